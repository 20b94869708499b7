// CUDA-core compute roofs of this GPU: FP64 and FP32 fused multiply-add throughput.
//
// The element kernels are not tensor-core work (12x12 and 30x30 element blocks), so the
// compute bound that matters beside HBM is the FP64 and FP32 FMA rate of the CUDA cores.
// Each thread runs kChains independent FMA chains for `iters` steps (enough independent
// work to cover the FMA latency at full occupancy) and folds them into one value that
// it stores, so nothing is dead code.  FLOPs per launch = 2 * kChains * iters * threads.
#include <cuda_runtime.h>
#include <stdint.h>

#include "psierra_b200.h"
#include "psx_common.cuh"

namespace {

constexpr int kChains = 8;
constexpr int kThreads = 256;

template <typename T>
__global__ void __launch_bounds__(kThreads) fma_kernel(int64_t iters, T a, T b, T* sink) {
  T x[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c) x[c] = (T)(threadIdx.x + c) * (T)1e-3;
  for (int64_t i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = fma(x[c], a, b);
  }
  T s = 0;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += x[c];
  sink[blockIdx.x * (int64_t)blockDim.x + threadIdx.x] = s;
}

}  // namespace

extern "C" int psx_fma_roof(int precision, int64_t iters, int blocks, void* sink, double* flops, void* stream) {
  if (iters <= 0 || blocks <= 0 || !sink || !flops) return PSX_ERR_ARG;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // a = 1 - 2^-20 and a small b keep every chain finite and away from denormals
  if (precision == PSX_FP64)
    fma_kernel<double><<<blocks, kThreads, 0, s>>>(iters, 1.0 - 0x1p-20, 1e-9, static_cast<double*>(sink));
  else if (precision == PSX_FP32_MIXED)
    fma_kernel<float><<<blocks, kThreads, 0, s>>>(iters, 1.0f - 0x1p-20f, 1e-9f, static_cast<float*>(sink));
  else
    return PSX_ERR_ARG;
  PSX_CUDA_CHECK_LAUNCH();
  *flops = 2.0 * kChains * (double)iters * (double)blocks * kThreads;
  return PSX_OK;
}

extern "C" int64_t psx_fma_roof_sink_bytes(int blocks) { return (int64_t)blocks * kThreads * 8; }
