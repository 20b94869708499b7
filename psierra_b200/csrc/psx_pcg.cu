// Preconditioned conjugate gradients on a CSR matrix (sm_100a).
//
// Restates the iteration of scipy.sparse.linalg.cg as the reference calls it from
// ConjugateGradientSolver.solve (psierra solver/sparse_linear_solver.py:37-68):
//   atol = max(atol, rtol ||b||);  r = b - A x
//   loop: if ||r|| < atol: converged
//         z = M^-1 r;  rho = r.z;  p = z (first) | p = z + (rho/rho_prev) p
//         q = A p;  alpha = rho / p.q;  x += alpha p;  r -= alpha q
// with the Jacobi preconditioner of the reference (1/diag where |diag| > 1e-14, else 1)
// or a 3x3 block-Jacobi preconditioner (inverse of each node's diagonal block).
//
// Three kernels per iteration: p-update, SpMV (+ p.q), and the fused x/r/z update
// (+ r.r, r.z).  Every dot product is reduced deterministically: each block reduces its
// share with a fixed tree and stores a partial; the last block to finish (atomic
// ticket) sums the partials in index order.  All scalars stay on the device; once
// converged (or broken down) every kernel returns immediately, so the host only checks
// the state every few iterations.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <mutex>

#include "psx_common.cuh"

namespace psx {
namespace {

constexpr int kBlock = 256;
// Five blocks per SM: the node-blocked SpMV (48 registers) fits five, and the PCG
// iteration on the 3.07M-element cube takes 0.153 ms instead of 0.157 with four; six
// (launch bounds capping 40 registers) measured 0.169 ms; prefetching the next node's
// row range one pass ahead, 0.157 ms.
constexpr int kGridMax = 148 * 5;
constexpr int kRowLanes = 8;  // lanes per CSR row in the SpMV

struct PcgScalars {
  double rho, rho_prev, pq, alpha, rr, bb, atol2;
  int32_t converged, breakdown, iters, first;
  uint32_t ticket[4];
};

struct PcgWork {
  double* r;
  double* z;
  double* p;
  double* q;
  double* minv;   // Jacobi: n; block-Jacobi: 9 per node
  double* partial;  // 3 * grid
  PcgScalars* s;
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Fixed-shape block reduction of up to 3 values; lane 0 of warp 0 gets the sums.
template <int NV>
__device__ __forceinline__ void block_sum(double v[NV]) {
  __shared__ double sm[NV][kBlock / 32];
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    const double t = warp_sum(v[i]);
    if (l == 0) sm[i][w] = t;
  }
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) v[i] = warp_sum(l < kBlock / 32 ? sm[i][l] : 0.0);
  }
  __syncthreads();
}

// Store this block's partial sums; the last block reduces all partials in index order
// and returns true (in thread 0) with the totals in `tot`.
template <int NV>
__device__ __forceinline__ bool last_block_total(double v[NV], double* partial, uint32_t* ticket, double tot[NV]) {
  block_sum<NV>(v);
  __shared__ bool s_last;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) partial[i * kGridMax + blockIdx.x] = v[i];
    __threadfence();
    s_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return false;
  __threadfence();
  double acc[NV];
#pragma unroll
  for (int i = 0; i < NV; ++i) acc[i] = 0.0;
  for (int bidx = threadIdx.x; bidx < (int)gridDim.x; bidx += kBlock)
#pragma unroll
    for (int i = 0; i < NV; ++i) acc[i] += __ldcg(partial + i * kGridMax + bidx);
  block_sum<NV>(acc);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) tot[i] = acc[i];
    *ticket = 0;
  }
  return threadIdx.x == 0;
}

__device__ __forceinline__ bool stopped(const PcgScalars* s) {
  return *(volatile const int32_t*)&s->converged || *(volatile const int32_t*)&s->breakdown;
}

// ---- preconditioner setup -----------------------------------------------------------
__global__ void jacobi_setup(int64_t n, const int32_t* __restrict__ indptr, const int32_t* __restrict__ indices,
                             const void* __restrict__ vals, int fp32, double* __restrict__ minv, int identity) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    int32_t lo = indptr[i], hi = indptr[i + 1] - 1;
    double d = 0.0;
    while (lo <= hi) {  // sorted column indices
      const int32_t mid = (lo + hi) >> 1;
      const int32_t c = indices[mid];
      if (c == i) {
        d = fp32 ? (double)static_cast<const float*>(vals)[mid] : static_cast<const double*>(vals)[mid];
        break;
      }
      if (c < i) lo = mid + 1; else hi = mid - 1;
    }
    minv[i] = identity ? 1.0 : (fabs(d) > 1e-14 ? 1.0 / d : 1.0);
  }
}

__device__ __forceinline__ double csr_at(const int32_t* indptr, const int32_t* indices, const void* vals, int fp32,
                                         int64_t row, int64_t col) {
  int32_t lo = indptr[row], hi = indptr[row + 1] - 1;
  while (lo <= hi) {
    const int32_t mid = (lo + hi) >> 1;
    const int32_t c = indices[mid];
    if (c == col) return fp32 ? (double)static_cast<const float*>(vals)[mid] : static_cast<const double*>(vals)[mid];
    if (c < col) lo = mid + 1; else hi = mid - 1;
  }
  return 0.0;
}

__global__ void bjacobi_setup(int64_t nodes, const int32_t* __restrict__ indptr, const int32_t* __restrict__ indices,
                              const void* __restrict__ vals, int fp32, double* __restrict__ binv,
                              PcgScalars* s) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nodes;
       i += (int64_t)gridDim.x * blockDim.x) {
    double B[3][3], Bi[3][3];
    for (int k = 0; k < 3; ++k)
      for (int m = 0; m < 3; ++m) B[k][m] = csr_at(indptr, indices, vals, fp32, 3 * i + k, 3 * i + m);
    const double det = inv3(B, Bi);
    const bool ok = fabs(det) > 1e-300 && isfinite(det);
    for (int k = 0; k < 3; ++k)
      for (int m = 0; m < 3; ++m) binv[9 * i + 3 * k + m] = ok ? Bi[k][m] : (k == m ? 1.0 : 0.0);
  }
}

// z = M^-1 r for element/node `i`.
template <bool BLOCK>
__device__ __forceinline__ void apply_prec(const PcgWork& w, int64_t i, double* __restrict__ z,
                                           const double* __restrict__ r) {
  if constexpr (BLOCK) {
    const double* B = w.minv + 9 * i;
    const double r0 = r[3 * i], r1 = r[3 * i + 1], r2 = r[3 * i + 2];
    z[3 * i] = B[0] * r0 + B[1] * r1 + B[2] * r2;
    z[3 * i + 1] = B[3] * r0 + B[4] * r1 + B[5] * r2;
    z[3 * i + 2] = B[6] * r0 + B[7] * r1 + B[8] * r2;
  } else {
    z[i] = w.minv[i] * r[i];
  }
}

// ---- SpMV: q = A p (8 lanes per row, fixed-order lane sums) and the p.q partials ------
template <typename VT>
__device__ __forceinline__ double spmv_row(int64_t n, int64_t row, int lane8, const int32_t* __restrict__ indptr,
                                           const int32_t* __restrict__ indices, const VT* __restrict__ vals,
                                           const double* __restrict__ x) {
  // rows past the end run the same shuffles with an empty range
  const int32_t j0 = row < n ? indptr[row] : 0, j1 = row < n ? indptr[row + 1] : 0;
  double acc = 0.0;
  for (int32_t j = j0 + lane8; j < j1; j += kRowLanes) acc += (double)vals[j] * __ldcg(x + indices[j]);
#pragma unroll
  for (int o = kRowLanes / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  return acc;
}

// Node-blocked CSR (PSX_PCG_NODAL): the three rows of node i have the same columns, in
// triples 3j, 3j+1, 3j+2 per neighbour j, and row 3i+k starts k * len after row 3i.  A
// quarter warp per node: lane l takes neighbours l, l + 8, ...; it reads the neighbour's
// column once (from row 3i), x once for the three rows, and the 3x3 block's values, then
// the three sums are reduced over the lane group in a fixed order.
// Scalar loads: the 8 lanes of a group read 24 consecutive values of a row per load
// instruction.  Loading each row segment and x triple as an aligned pair plus a scalar
// (9 instead of 13 loads per neighbour) measured slower: 0.194 instead of 0.155 ms.
// Unrolling the neighbour loop by 2 or 4 did too: 0.171 and 0.158 instead of 0.156 ms.
// The matrix values and column indices are read once per SpMV, while every neighbour of
// a node gathers its x triple: the matrix is loaded with the streaming (evict-first)
// hint, so that it does not push x out of L2.  PCG iteration 0.152 -> 0.146 ms; an L2
// evict_last policy on the x loads as well measured 0.148 ms.
constexpr int kNodeLanes = 8;  // PCG iteration on the 3.07M-element cube: 0.157 ms (16 lanes 0.176, 4 lanes 0.165)
template <typename VT>
__device__ __forceinline__ void spmv_node(int64_t nodes, int64_t node, int lane16, const int32_t* __restrict__ indptr,
                                          const int32_t* __restrict__ indices, const VT* __restrict__ vals,
                                          const double* __restrict__ x, double out[3]) {
  // nodes past the end run the same shuffles with an empty range
  int32_t r0 = 0, len = 0;
  if (node < nodes) {
    r0 = indptr[3 * node];
    len = indptr[3 * node + 1] - r0;
  }
  double a0 = 0.0, a1 = 0.0, a2 = 0.0;
  for (int32_t b3 = 3 * lane16; b3 < len; b3 += 3 * kNodeLanes) {
    const int32_t c = __ldcs(indices + r0 + b3);
    const double x0 = __ldcg(x + c), x1 = __ldcg(x + c + 1), x2 = __ldcg(x + c + 2);
    const VT* v0 = vals + r0 + b3;
    const VT* v1 = v0 + len;
    const VT* v2 = v1 + len;
    a0 += (double)__ldcs(v0) * x0 + (double)__ldcs(v0 + 1) * x1 + (double)__ldcs(v0 + 2) * x2;
    a1 += (double)__ldcs(v1) * x0 + (double)__ldcs(v1 + 1) * x1 + (double)__ldcs(v1 + 2) * x2;
    a2 += (double)__ldcs(v2) * x0 + (double)__ldcs(v2 + 1) * x1 + (double)__ldcs(v2 + 2) * x2;
  }
#pragma unroll
  for (int o = kNodeLanes / 2; o > 0; o >>= 1) {
    a0 += __shfl_xor_sync(0xffffffffu, a0, o);
    a1 += __shfl_xor_sync(0xffffffffu, a1, o);
    a2 += __shfl_xor_sync(0xffffffffu, a2, o);
  }
  out[0] = a0;
  out[1] = a1;
  out[2] = a2;
}

// r = b - A x, z = M^-1 r, and the sums r.r, r.z, b.b (setup of the iteration).
template <typename VT, bool BLOCK, bool NODAL>
__global__ void __launch_bounds__(kBlock) pcg_init_residual(int64_t n, const int32_t* __restrict__ indptr,
                                                            const int32_t* __restrict__ indices,
                                                            const VT* __restrict__ vals, const double* __restrict__ b,
                                                            const double* __restrict__ x, PcgWork w) {
  if constexpr (NODAL) {
    const int lane16 = threadIdx.x & (kNodeLanes - 1);
    const int64_t nodes = n / 3, per_pass = (int64_t)gridDim.x * (kBlock / kNodeLanes);
    for (int64_t node0 = blockIdx.x * (int64_t)(kBlock / kNodeLanes); node0 < nodes; node0 += per_pass) {
      const int64_t node = node0 + threadIdx.x / kNodeLanes;
      double ax[3];
      spmv_node<VT>(nodes, node, lane16, indptr, indices, vals, x, ax);
      if (node < nodes && lane16 == 0)
        for (int k = 0; k < 3; ++k) w.r[3 * node + k] = b[3 * node + k] - ax[k];
    }
    return;
  }
  const int lane8 = threadIdx.x & (kRowLanes - 1);
  const int64_t rows_per_pass = (int64_t)gridDim.x * (kBlock / kRowLanes);
  for (int64_t row0 = blockIdx.x * (int64_t)(kBlock / kRowLanes); row0 < n; row0 += rows_per_pass) {
    const int64_t row = row0 + threadIdx.x / kRowLanes;
    const double ax = spmv_row<VT>(n, row, lane8, indptr, indices, vals, x);
    if (row < n && lane8 == 0) w.r[row] = b[row] - ax;
  }
}

template <bool BLOCK>
__global__ void __launch_bounds__(kBlock) pcg_init_dots(int64_t n, const double* __restrict__ b, PcgWork w,
                                                        double rtol, double atol) {
  double v[3] = {0.0, 0.0, 0.0};
  const int64_t units = BLOCK ? n / 3 : n;
  for (int64_t i = blockIdx.x * (int64_t)kBlock + threadIdx.x; i < units; i += (int64_t)gridDim.x * kBlock) {
    apply_prec<BLOCK>(w, i, w.z, w.r);
    const int nd = BLOCK ? 3 : 1;
    for (int k = 0; k < nd; ++k) {
      const int64_t d = BLOCK ? 3 * i + k : i;
      v[0] += w.r[d] * w.r[d];
      v[1] += w.r[d] * w.z[d];
      v[2] += b[d] * b[d];
    }
  }
  double tot[3];
  if (last_block_total<3>(v, w.partial, &w.s->ticket[0], tot)) {
    PcgScalars* s = w.s;
    s->rr = tot[0];
    s->rho = tot[1];
    s->bb = tot[2];
    const double a = fmax(atol, rtol * sqrt(tot[2]));
    s->atol2 = a * a;
    s->iters = 0;
    s->first = 1;
    s->breakdown = 0;
    // scipy returns x = b (= 0 for x0 = 0 handled by the caller) when ||b|| == 0
    s->converged = (tot[2] == 0.0 || sqrt(tot[0]) < a) ? 1 : 0;
  }
}

// p = z (first iteration) or p = z + beta p
template <bool BLOCK>
__global__ void __launch_bounds__(kBlock) pcg_update_p(int64_t n, PcgWork w) {
  const PcgScalars* s = w.s;
  if (stopped(s)) return;
  const bool first = s->first != 0;
  const double beta = first ? 0.0 : s->rho / s->rho_prev;
  for (int64_t i = blockIdx.x * (int64_t)kBlock + threadIdx.x; i < n; i += (int64_t)gridDim.x * kBlock)
    w.p[i] = first ? w.z[i] : w.z[i] + beta * w.p[i];
}

// q = A p and p.q -> alpha = rho / p.q
template <typename VT, bool NODAL>
__global__ void __launch_bounds__(kBlock) pcg_spmv(int64_t n, const int32_t* __restrict__ indptr,
                                                   const int32_t* __restrict__ indices, const VT* __restrict__ vals,
                                                   PcgWork w) {
  if (stopped(w.s)) return;
  double v[1] = {0.0};
  if constexpr (NODAL) {
    const int lane16 = threadIdx.x & (kNodeLanes - 1);
    const int64_t nodes = n / 3, per_pass = (int64_t)gridDim.x * (kBlock / kNodeLanes);
    for (int64_t node0 = blockIdx.x * (int64_t)(kBlock / kNodeLanes); node0 < nodes; node0 += per_pass) {
      const int64_t node = node0 + threadIdx.x / kNodeLanes;
      double q[3];
      spmv_node<VT>(nodes, node, lane16, indptr, indices, vals, w.p, q);
      if (node < nodes && lane16 == 0)
        for (int k = 0; k < 3; ++k) {
          w.q[3 * node + k] = q[k];
          v[0] += w.p[3 * node + k] * q[k];
        }
    }
  } else {
    const int lane8 = threadIdx.x & (kRowLanes - 1);
    const int64_t rows_per_pass = (int64_t)gridDim.x * (kBlock / kRowLanes);
    for (int64_t row0 = blockIdx.x * (int64_t)(kBlock / kRowLanes); row0 < n; row0 += rows_per_pass) {
      const int64_t row = row0 + threadIdx.x / kRowLanes;
      const double q = spmv_row<VT>(n, row, lane8, indptr, indices, vals, w.p);
      if (row < n && lane8 == 0) {
        w.q[row] = q;
        v[0] += w.p[row] * q;
      }
    }
  }
  double tot[1];
  if (last_block_total<1>(v, w.partial, &w.s->ticket[1], tot)) {
    PcgScalars* s = w.s;
    s->pq = tot[0];
    if (!(tot[0] != 0.0) || !isfinite(tot[0])) s->breakdown = 1;
    s->alpha = s->rho / tot[0];
  }
}

// x += alpha p; r -= alpha q; z = M^-1 r; r.r and r.z for the next iteration.
template <bool BLOCK>
__global__ void __launch_bounds__(kBlock) pcg_update_xr(int64_t n, double* __restrict__ x, PcgWork w,
                                                        int32_t maxiter) {
  PcgScalars* s = w.s;
  if (stopped(s)) return;
  const double alpha = s->alpha;
  double v[2] = {0.0, 0.0};
  const int64_t units = BLOCK ? n / 3 : n;
  for (int64_t i = blockIdx.x * (int64_t)kBlock + threadIdx.x; i < units; i += (int64_t)gridDim.x * kBlock) {
    const int nd = BLOCK ? 3 : 1;
    for (int k = 0; k < nd; ++k) {
      const int64_t d = BLOCK ? 3 * i + k : i;
      x[d] += alpha * w.p[d];
      w.r[d] -= alpha * w.q[d];
    }
    apply_prec<BLOCK>(w, i, w.z, w.r);
    for (int k = 0; k < nd; ++k) {
      const int64_t d = BLOCK ? 3 * i + k : i;
      v[0] += w.r[d] * w.r[d];
      v[1] += w.r[d] * w.z[d];
    }
  }
  double tot[2];
  if (last_block_total<2>(v, w.partial, &w.s->ticket[2], tot)) {
    s->rho_prev = s->rho;
    s->rr = tot[0];
    s->rho = tot[1];
    s->first = 0;
    s->iters += 1;
    // scipy checks the residual at the top of each of its maxiter iterations, so a
    // residual reached by the last allowed update still reports non-convergence
    if (!isfinite(tot[0])) s->breakdown = 1;
    else if (s->iters >= maxiter) s->breakdown = 2;
    else if (tot[0] < s->atol2) s->converged = 1;
  }
}

// ---- two-level preconditioner: rigid-body modes per aggregate --------------------------
// P^T w for aggregate a: translations sum w_i, rotations sum d_i x w_i (the column of
// rotation e at node i is e x d_i, and (e x d).w = e.(d x w)).  One warp per aggregate,
// lane sums in a fixed order.
__global__ void __launch_bounds__(kBlock) coarse_restrict_kernel(psx_coarse_t c, const double* __restrict__ w,
                                                                 double* __restrict__ out, const PcgScalars* s) {
  if (s && stopped(s)) return;
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (kBlock / 32);
  for (int64_t a = blockIdx.x * (int64_t)(kBlock / 32) + (threadIdx.x >> 5); a < c.n_agg; a += warps) {
    double t[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int32_t k = c.agg_ptr[a] + lane; k < c.agg_ptr[a + 1]; k += 32) {
      const int64_t i = c.agg_nodes[k];
      double v[3];
#pragma unroll
      for (int m = 0; m < 3; ++m) v[m] = c.fixed[3 * i + m] ? 0.0 : w[3 * i + m];
      const double dx = c.d[3 * i], dy = c.d[3 * i + 1], dz = c.d[3 * i + 2];
      t[0] += v[0];
      t[1] += v[1];
      t[2] += v[2];
      t[3] += dy * v[2] - dz * v[1];
      t[4] += dz * v[0] - dx * v[2];
      t[5] += dx * v[1] - dy * v[0];
    }
#pragma unroll
    for (int m = 0; m < 6; ++m) t[m] = warp_sum(t[m]);
    if (lane == 0)
#pragma unroll
      for (int m = 0; m < 6; ++m) out[6 * a + m] = t[m];
  }
}

// yc = A_c^-1 rc per block (one thread block each, a warp per row, lane sums in a fixed
// order); the block's right-hand side is staged in shared memory.
__global__ void __launch_bounds__(kBlock) coarse_gemv_kernel(psx_coarse_t c, const PcgScalars* s) {
  if (s && stopped(s)) return;
  extern __shared__ double s_rhs[];
  const int32_t a0 = c.block_agg[blockIdx.x];
  const int m = 6 * (c.block_agg[blockIdx.x + 1] - a0);
  if (m < 0 || m > c.nc) return;  // inconsistent block sizes: stay inside the staged right-hand side
  for (int k = threadIdx.x; k < m; k += kBlock) s_rhs[k] = c.rc[6 * (int64_t)a0 + k];
  __syncthreads();
  const double* A = c.ainv + (int64_t)blockIdx.x * c.nc * c.nc;
  const int lane = threadIdx.x & 31;
  for (int r = threadIdx.x >> 5; r < m; r += kBlock / 32) {
    double acc = 0.0;
    for (int k = lane; k < m; k += 32) acc += A[(int64_t)r * c.nc + k] * s_rhs[k];
    acc = warp_sum(acc);
    if (lane == 0) c.yc[6 * (int64_t)a0 + r] = acc;
  }
}

// v = sum of column `mode` of P over the aggregates of colour `color`.
__global__ void coarse_probe_kernel(psx_coarse_t c, const int32_t* __restrict__ color_of, int32_t color, int32_t mode,
                                    double* __restrict__ v) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < c.n_nodes; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t a = c.node_agg[i];
    double col[3] = {0.0, 0.0, 0.0};
    if (a >= 0 && color_of[a] == color) {
      const double dx = c.d[3 * i], dy = c.d[3 * i + 1], dz = c.d[3 * i + 2];
      if (mode < 3) {
        col[mode] = 1.0;
      } else if (mode == 3) {  // e_x x d
        col[1] = -dz;
        col[2] = dy;
      } else if (mode == 4) {  // e_y x d
        col[0] = dz;
        col[2] = -dx;
      } else {  // e_z x d
        col[0] = -dy;
        col[1] = dx;
      }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) v[3 * i + k] = c.fixed[3 * i + k] ? 0.0 : col[k];
  }
}

// x += alpha p; r -= alpha q (the two-level iteration forms z after the coarse solve)
__global__ void __launch_bounds__(kBlock) pcg_update_xr_only(int64_t n, double* __restrict__ x, PcgWork w) {
  if (stopped(w.s)) return;
  const double alpha = w.s->alpha;
  for (int64_t i = blockIdx.x * (int64_t)kBlock + threadIdx.x; i < n; i += (int64_t)gridDim.x * kBlock) {
    x[i] += alpha * w.p[i];
    w.r[i] -= alpha * w.q[i];
  }
}

// z = B^-1 r + P yc per node, with r.r and r.z (and b.b on the first call) and the
// bookkeeping of pcg_init_dots (INIT) or pcg_update_xr.
template <bool INIT>
__global__ void __launch_bounds__(kBlock) pcg_coarse_z(int64_t n, const double* __restrict__ b, PcgWork w,
                                                       psx_coarse_t c, double rtol, double atol, int32_t maxiter) {
  if (!INIT && stopped(w.s)) return;
  double v[3] = {0.0, 0.0, 0.0};
  for (int64_t i = blockIdx.x * (int64_t)kBlock + threadIdx.x; i < n / 3; i += (int64_t)gridDim.x * kBlock) {
    apply_prec<true>(w, i, w.z, w.r);
    const int32_t a = c.node_agg[i];
    if (a >= 0) {
      const double* y = c.yc + 6 * (int64_t)a;
      const double dx = c.d[3 * i], dy = c.d[3 * i + 1], dz = c.d[3 * i + 2];
      const double add[3] = {y[0] + (y[4] * dz - y[5] * dy), y[1] + (y[5] * dx - y[3] * dz),
                             y[2] + (y[3] * dy - y[4] * dx)};
#pragma unroll
      for (int k = 0; k < 3; ++k)
        if (!c.fixed[3 * i + k]) w.z[3 * i + k] += add[k];
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const int64_t d = 3 * i + k;
      v[0] += w.r[d] * w.r[d];
      v[1] += w.r[d] * w.z[d];
      if constexpr (INIT) v[2] += b[d] * b[d];
    }
  }
  PcgScalars* s = w.s;
  if constexpr (INIT) {
    double tot[3];
    if (last_block_total<3>(v, w.partial, &s->ticket[0], tot)) {
      s->rr = tot[0];
      s->rho = tot[1];
      s->bb = tot[2];
      const double a = fmax(atol, rtol * sqrt(tot[2]));
      s->atol2 = a * a;
      s->iters = 0;
      s->first = 1;
      s->breakdown = 0;
      s->converged = (tot[2] == 0.0 || sqrt(tot[0]) < a) ? 1 : 0;
    }
  } else {
    double tot[2];
    if (last_block_total<2>(v, w.partial, &s->ticket[2], tot)) {
      s->rho_prev = s->rho;
      s->rr = tot[0];
      s->rho = tot[1];
      s->first = 0;
      s->iters += 1;
      if (!isfinite(tot[0])) s->breakdown = 1;
      else if (s->iters >= maxiter) s->breakdown = 2;
      else if (tot[0] < s->atol2) s->converged = 1;
    }
  }
}

__global__ void pcg_report(const PcgScalars* s, Status* st) {
  st->iters = s->iters;
  st->flags = s->converged ? 0 : (s->breakdown == 2 ? 2 : 4);
  st->value = sqrt(s->rr);
}

size_t up256(size_t b) { return (b + 255) / 256 * 256; }

int layout(int64_t n, int precond, void* work, PcgWork* w, int64_t* bytes) {
  const size_t vec = up256(sizeof(double) * n);
  const size_t mv = precond == PSX_PRECOND_BJACOBI ? up256(sizeof(double) * 3 * n) : vec;
  const size_t part = up256(sizeof(double) * 3 * kGridMax);
  const size_t sc = up256(sizeof(PcgScalars));
  *bytes = (int64_t)(4 * vec + mv + part + sc);
  if (!work) return PSX_OK;
  if (reinterpret_cast<uintptr_t>(work) & 255) return PSX_ERR_ARG;
  char* c = static_cast<char*>(work);
  w->r = reinterpret_cast<double*>(c);
  w->z = reinterpret_cast<double*>(c + vec);
  w->p = reinterpret_cast<double*>(c + 2 * vec);
  w->q = reinterpret_cast<double*>(c + 3 * vec);
  w->minv = reinterpret_cast<double*>(c + 4 * vec);
  w->partial = reinterpret_cast<double*>(c + 4 * vec + mv);
  w->s = reinterpret_cast<PcgScalars*>(c + 4 * vec + mv + part);
  return PSX_OK;
}

template <typename VT, bool BLOCK, bool NODAL>
int run_pcg(int64_t n, const int32_t* indptr, const int32_t* indices, const VT* vals, const double* b, double* x,
            double rtol, double atol, int32_t maxiter, const PcgWork& w, Status* st, cudaStream_t s,
            int identity, bool host_checks) {
  const int grid_vec = (int)std::min<int64_t>(kGridMax, (n + kBlock - 1) / kBlock);
  const int grid_row = NODAL ? (int)std::min<int64_t>(kGridMax, (n / 3 + kBlock / kNodeLanes - 1) / (kBlock / kNodeLanes))
                             : (int)std::min<int64_t>(kGridMax, (n + kBlock / kRowLanes - 1) / (kBlock / kRowLanes));
  if (cudaMemsetAsync(w.s, 0, sizeof(PcgScalars), s) != cudaSuccess) return PSX_ERR_CUDA;
  if (BLOCK)
    bjacobi_setup<<<grid_vec, kBlock, 0, s>>>(n / 3, indptr, indices, vals, sizeof(VT) == 4, w.minv, w.s);
  else
    jacobi_setup<<<grid_vec, kBlock, 0, s>>>(n, indptr, indices, vals, sizeof(VT) == 4, w.minv, identity);
  pcg_init_residual<VT, BLOCK, NODAL><<<grid_row, kBlock, 0, s>>>(n, indptr, indices, vals, b, x, w);
  pcg_init_dots<BLOCK><<<grid_vec, kBlock, 0, s>>>(n, b, w, rtol, atol);
  PSX_CUDA_CHECK_LAUNCH();
  // iterate in batches; every kernel is a no-op once the state is converged or broken down
  PcgScalars host;
  int32_t done = 0;
  constexpr int kBatchIters = 16;
  while (done < maxiter) {
    const int32_t batch = std::min<int32_t>(kBatchIters, maxiter - done);
    for (int32_t k = 0; k < batch; ++k) {
      pcg_update_p<BLOCK><<<grid_vec, kBlock, 0, s>>>(n, w);
      pcg_spmv<VT, NODAL><<<grid_row, kBlock, 0, s>>>(n, indptr, indices, vals, w);
      pcg_update_xr<BLOCK><<<grid_vec, kBlock, 0, s>>>(n, x, w, maxiter);
    }
    PSX_CUDA_CHECK_LAUNCH();
    done += batch;
    if (!host_checks) continue;  // fixed trip count, nothing read back (stream-capturable)
    if (cudaMemcpyAsync(&host, w.s, sizeof(PcgScalars), cudaMemcpyDeviceToHost, s) != cudaSuccess)
      return PSX_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return PSX_ERR_CUDA;
    if (host.converged || host.breakdown) break;
  }
  pcg_report<<<1, 1, 0, s>>>(w.s, st);
  PSX_CUDA_CHECK_LAUNCH();
  return PSX_OK;
}

constexpr int kCoarseMaxNc = 6144;  // coarse size per block: its right-hand side fits 48 KB of shared memory

// The two-level iteration: block-Jacobi plus the coarse correction, six kernels per
// iteration (p update, SpMV + p.q, x/r update, restriction, coarse solve, z + dots).
template <typename VT, bool NODAL>
int run_pcg_coarse(int64_t n, const int32_t* indptr, const int32_t* indices, const VT* vals, const double* b,
                   double* x, double rtol, double atol, int32_t maxiter, const PcgWork& w, const psx_coarse_t& c,
                   Status* st, cudaStream_t s, bool host_checks) {
  const int grid_vec = (int)std::min<int64_t>(kGridMax, (n + kBlock - 1) / kBlock);
  const int grid_nodes = (int)std::min<int64_t>(kGridMax, (n / 3 + kBlock - 1) / kBlock);
  const int grid_row = NODAL ? (int)std::min<int64_t>(kGridMax, (n / 3 + kBlock / kNodeLanes - 1) / (kBlock / kNodeLanes))
                             : (int)std::min<int64_t>(kGridMax, (n + kBlock / kRowLanes - 1) / (kBlock / kRowLanes));
  const int grid_agg = (int)std::min<int64_t>(kGridMax, (c.n_agg + kBlock / 32 - 1) / (kBlock / 32));
  const size_t smem = sizeof(double) * (size_t)c.nc;
  if (cudaMemsetAsync(w.s, 0, sizeof(PcgScalars), s) != cudaSuccess) return PSX_ERR_CUDA;
  bjacobi_setup<<<grid_vec, kBlock, 0, s>>>(n / 3, indptr, indices, vals, sizeof(VT) == 4, w.minv, w.s);
  pcg_init_residual<VT, true, NODAL><<<grid_row, kBlock, 0, s>>>(n, indptr, indices, vals, b, x, w);
  coarse_restrict_kernel<<<grid_agg, kBlock, 0, s>>>(c, w.r, c.rc, nullptr);
  coarse_gemv_kernel<<<c.n_blocks, kBlock, smem, s>>>(c, nullptr);
  pcg_coarse_z<true><<<grid_nodes, kBlock, 0, s>>>(n, b, w, c, rtol, atol, maxiter);
  PSX_CUDA_CHECK_LAUNCH();
  PcgScalars host;
  int32_t done = 0;
  constexpr int kBatchIters = 16;
  while (done < maxiter) {
    const int32_t batch = std::min<int32_t>(kBatchIters, maxiter - done);
    for (int32_t k = 0; k < batch; ++k) {
      pcg_update_p<true><<<grid_vec, kBlock, 0, s>>>(n, w);
      pcg_spmv<VT, NODAL><<<grid_row, kBlock, 0, s>>>(n, indptr, indices, vals, w);
      pcg_update_xr_only<<<grid_vec, kBlock, 0, s>>>(n, x, w);
      coarse_restrict_kernel<<<grid_agg, kBlock, 0, s>>>(c, w.r, c.rc, w.s);
      coarse_gemv_kernel<<<c.n_blocks, kBlock, smem, s>>>(c, w.s);
      pcg_coarse_z<false><<<grid_nodes, kBlock, 0, s>>>(n, b, w, c, rtol, atol, maxiter);
    }
    PSX_CUDA_CHECK_LAUNCH();
    done += batch;
    if (!host_checks) continue;
    if (cudaMemcpyAsync(&host, w.s, sizeof(PcgScalars), cudaMemcpyDeviceToHost, s) != cudaSuccess)
      return PSX_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return PSX_ERR_CUDA;
    if (host.converged || host.breakdown) break;
  }
  pcg_report<<<1, 1, 0, s>>>(w.s, st);
  PSX_CUDA_CHECK_LAUNCH();
  return PSX_OK;
}

bool coarse_ok(const psx_coarse_t* c) {
  return c && c->n_nodes > 0 && c->n_agg > 0 && c->node_agg && c->agg_ptr && c->agg_nodes && c->d && c->fixed &&
         c->n_blocks > 0 && c->nc > 0 && c->nc <= kCoarseMaxNc && c->block_agg && c->ainv && c->rc && c->yc;
}

// ---- batched CG: one independent CG per segment of a block-diagonal system -----------
// The unknowns of segment s are [off[s], off[s+1]) (whole nodes); each segment has its
// own step lengths, residual test and iteration count, so a batch of meshes solved as
// one system converges instance by instance, at each instance's own rate, instead of
// at the rate of the worst-conditioned instance (which shared step lengths give).  The
// per-segment dot products are reduced by one thread block per segment in a fixed
// order.
struct SegScalars {
  double rho, rho_prev, alpha, rr, bb, atol2;
  int32_t state;  // 0 running, 1 converged, 2 iteration limit, 4 breakdown
  int32_t iters, first, pad;
};

struct BatchArgs {
  int32_t n_seg;
  const int64_t* off;     // n_seg + 1 unknown offsets (multiples of 3)
  const int32_t* node_seg;  // segment of each node
  SegScalars* seg;
};

// z = B^-1 r (+ P yc) for every node of a running segment
template <bool COARSE>
__global__ void __launch_bounds__(kBlock) bpcg_precond(int64_t n, PcgWork w, BatchArgs ba, psx_coarse_t c) {
  for (int64_t i = blockIdx.x * (int64_t)kBlock + threadIdx.x; i < n / 3; i += (int64_t)gridDim.x * kBlock) {
    if (ba.seg[ba.node_seg[i]].state) continue;
    apply_prec<true>(w, i, w.z, w.r);
    if constexpr (COARSE) {
      const int32_t a = c.node_agg[i];
      if (a >= 0) {
        const double* y = c.yc + 6 * (int64_t)a;
        const double dx = c.d[3 * i], dy = c.d[3 * i + 1], dz = c.d[3 * i + 2];
        const double add[3] = {y[0] + (y[4] * dz - y[5] * dy), y[1] + (y[5] * dx - y[3] * dz),
                               y[2] + (y[3] * dy - y[4] * dx)};
#pragma unroll
        for (int k = 0; k < 3; ++k)
          if (!c.fixed[3 * i + k]) w.z[3 * i + k] += add[k];
      }
    }
  }
}

// Per-segment dot products, one block per segment.  KIND 0: initial (r.r, r.z, b.b);
// 1: p.q -> alpha; 2: (r.r, r.z) -> the next iteration's scalars and the residual test.
template <int KIND>
__global__ void __launch_bounds__(kBlock) bpcg_segdots(const double* __restrict__ b, PcgWork w, BatchArgs ba,
                                                        double rtol, double atol, int32_t maxiter) {
  SegScalars* s = ba.seg + blockIdx.x;
  if (KIND != 0 && s->state) return;
  const int64_t d0 = ba.off[blockIdx.x], d1 = ba.off[blockIdx.x + 1];
  double v[3] = {0.0, 0.0, 0.0};
  for (int64_t d = d0 + threadIdx.x; d < d1; d += kBlock) {
    if constexpr (KIND == 1) {
      v[0] += w.p[d] * w.q[d];
    } else {
      v[0] += w.r[d] * w.r[d];
      v[1] += w.r[d] * w.z[d];
      if constexpr (KIND == 0) v[2] += b[d] * b[d];
    }
  }
  block_sum<3>(v);
  if (threadIdx.x != 0) return;
  if constexpr (KIND == 0) {
    s->rr = v[0];
    s->rho = v[1];
    s->bb = v[2];
    const double a = fmax(atol, rtol * sqrt(v[2]));
    s->atol2 = a * a;
    s->iters = 0;
    s->first = 1;
    s->state = (v[2] == 0.0 || sqrt(v[0]) < a) ? 1 : 0;
  } else if constexpr (KIND == 1) {
    if (!(v[0] != 0.0) || !isfinite(v[0])) {
      s->state = 4;
      s->alpha = 0.0;
    } else {
      s->alpha = s->rho / v[0];
    }
  } else {
    s->rho_prev = s->rho;
    s->rr = v[0];
    s->rho = v[1];
    s->first = 0;
    s->iters += 1;
    if (!isfinite(v[0])) s->state = 4;
    else if (v[0] < s->atol2) s->state = 1;
    else if (s->iters >= maxiter) s->state = 2;
  }
}

__global__ void __launch_bounds__(kBlock) bpcg_update_p(int64_t n, PcgWork w, BatchArgs ba) {
  for (int64_t i = blockIdx.x * (int64_t)kBlock + threadIdx.x; i < n; i += (int64_t)gridDim.x * kBlock) {
    const SegScalars* s = ba.seg + ba.node_seg[i / 3];
    if (s->state) continue;
    w.p[i] = s->first ? w.z[i] : w.z[i] + (s->rho / s->rho_prev) * w.p[i];
  }
}

__global__ void __launch_bounds__(kBlock) bpcg_update_xr(int64_t n, double* __restrict__ x, PcgWork w, BatchArgs ba) {
  for (int64_t i = blockIdx.x * (int64_t)kBlock + threadIdx.x; i < n; i += (int64_t)gridDim.x * kBlock) {
    const SegScalars* s = ba.seg + ba.node_seg[i / 3];
    if (s->state) continue;
    x[i] += s->alpha * w.p[i];
    w.r[i] -= s->alpha * w.q[i];
  }
}

// q = A p over the whole system (the blocks of finished segments compute on a frozen p)
template <typename VT, bool NODAL>
__global__ void __launch_bounds__(kBlock) bpcg_spmv(int64_t n, const int32_t* __restrict__ indptr,
                                                    const int32_t* __restrict__ indices, const VT* __restrict__ vals,
                                                    PcgWork w) {
  if constexpr (NODAL) {
    const int lane16 = threadIdx.x & (kNodeLanes - 1);
    const int64_t nodes = n / 3, per_pass = (int64_t)gridDim.x * (kBlock / kNodeLanes);
    for (int64_t node0 = blockIdx.x * (int64_t)(kBlock / kNodeLanes); node0 < nodes; node0 += per_pass) {
      const int64_t node = node0 + threadIdx.x / kNodeLanes;
      double q[3];
      spmv_node<VT>(nodes, node, lane16, indptr, indices, vals, w.p, q);
      if (node < nodes && lane16 == 0)
        for (int k = 0; k < 3; ++k) w.q[3 * node + k] = q[k];
    }
  } else {
    const int lane8 = threadIdx.x & (kRowLanes - 1);
    const int64_t rows_per_pass = (int64_t)gridDim.x * (kBlock / kRowLanes);
    for (int64_t row0 = blockIdx.x * (int64_t)(kBlock / kRowLanes); row0 < n; row0 += rows_per_pass) {
      const int64_t row = row0 + threadIdx.x / kRowLanes;
      const double q = spmv_row<VT>(n, row, lane8, indptr, indices, vals, w.p);
      if (row < n && lane8 == 0) w.q[row] = q;
    }
  }
}

__global__ void bpcg_report(BatchArgs ba, Status* st, int32_t* seg_iters) {
  int32_t most = 0, flags = 0;
  double rr = 0.0;
  for (int32_t s = 0; s < ba.n_seg; ++s) {
    const SegScalars& g = ba.seg[s];
    most = max(most, g.iters);
    if (g.state != 1) flags |= g.state == 2 ? 2 : 4;
    rr += g.rr;
    if (seg_iters) seg_iters[s] = g.state == 1 ? g.iters : -g.iters - 1;
  }
  st->iters = most;
  st->flags = flags;
  st->value = sqrt(rr);
}

template <typename VT, bool NODAL, bool COARSE>
int run_pcg_batched(int64_t n, const int32_t* indptr, const int32_t* indices, const VT* vals, const double* b,
                    double* x, double rtol, double atol, int32_t maxiter, const PcgWork& w, const BatchArgs& ba,
                    const psx_coarse_t& c, Status* st, int32_t* seg_iters, cudaStream_t s) {
  const int grid_vec = (int)std::min<int64_t>(kGridMax, (n + kBlock - 1) / kBlock);
  const int grid_nodes = (int)std::min<int64_t>(kGridMax, (n / 3 + kBlock - 1) / kBlock);
  const int grid_row = NODAL ? (int)std::min<int64_t>(kGridMax, (n / 3 + kBlock / kNodeLanes - 1) / (kBlock / kNodeLanes))
                             : (int)std::min<int64_t>(kGridMax, (n + kBlock / kRowLanes - 1) / (kBlock / kRowLanes));
  const int grid_agg = COARSE ? (int)std::min<int64_t>(kGridMax, (c.n_agg + kBlock / 32 - 1) / (kBlock / 32)) : 1;
  const size_t smem = COARSE ? sizeof(double) * (size_t)c.nc : 0;
  if (cudaMemsetAsync(ba.seg, 0, sizeof(SegScalars) * ba.n_seg, s) != cudaSuccess) return PSX_ERR_CUDA;
  bjacobi_setup<<<grid_vec, kBlock, 0, s>>>(n / 3, indptr, indices, vals, sizeof(VT) == 4, w.minv, w.s);
  pcg_init_residual<VT, true, NODAL><<<grid_row, kBlock, 0, s>>>(n, indptr, indices, vals, b, x, w);
  auto precond = [&]() {
    if constexpr (COARSE) {
      coarse_restrict_kernel<<<grid_agg, kBlock, 0, s>>>(c, w.r, c.rc, nullptr);
      coarse_gemv_kernel<<<c.n_blocks, kBlock, smem, s>>>(c, nullptr);
    }
    bpcg_precond<COARSE><<<grid_nodes, kBlock, 0, s>>>(n, w, ba, c);
  };
  precond();
  bpcg_segdots<0><<<ba.n_seg, kBlock, 0, s>>>(b, w, ba, rtol, atol, maxiter);
  PSX_CUDA_CHECK_LAUNCH();
  for (int32_t k = 0; k < maxiter; ++k) {
    bpcg_update_p<<<grid_vec, kBlock, 0, s>>>(n, w, ba);
    bpcg_spmv<VT, NODAL><<<grid_row, kBlock, 0, s>>>(n, indptr, indices, vals, w);
    bpcg_segdots<1><<<ba.n_seg, kBlock, 0, s>>>(b, w, ba, rtol, atol, maxiter);
    bpcg_update_xr<<<grid_vec, kBlock, 0, s>>>(n, x, w, ba);
    precond();
    bpcg_segdots<2><<<ba.n_seg, kBlock, 0, s>>>(b, w, ba, rtol, atol, maxiter);
    if ((k & 15) == 15) PSX_CUDA_CHECK_LAUNCH();
  }
  bpcg_report<<<1, 1, 0, s>>>(ba, st, seg_iters);
  PSX_CUDA_CHECK_LAUNCH();
  return PSX_OK;
}

}  // namespace
}  // namespace psx

extern "C" int psx_pcg_work_bytes(int64_t n, int precond, int64_t* bytes) {
  precond &= ~PSX_PCG_NODAL;
  if (n <= 0 || !bytes || precond < PSX_PRECOND_NONE || precond > PSX_PRECOND_BJACOBI) return PSX_ERR_ARG;
  if (precond == PSX_PRECOND_BJACOBI && n % 3) return PSX_ERR_ARG;
  psx::PcgWork w;
  return psx::layout(n, precond, nullptr, &w, bytes);
}

namespace {
int pcg_entry(int64_t n, const int32_t* indptr, const int32_t* indices, const void* values, int value_precision,
              const double* b, double* x, double rtol, double atol, int32_t maxiter, int precond, void* work,
              int64_t work_bytes, void* status, void* stream, bool host_checks) {
  using namespace psx;
  if (n <= 0 || !indptr || !indices || !values || !b || !x || !work || !status || maxiter < 0) return PSX_ERR_ARG;
  const bool nodal = (precond & PSX_PCG_NODAL) != 0;
  precond &= ~PSX_PCG_NODAL;
  if (nodal && n % 3) return PSX_ERR_ARG;
  if (precond < PSX_PRECOND_NONE || precond > PSX_PRECOND_BJACOBI) return PSX_ERR_ARG;
  if (precond == PSX_PRECOND_BJACOBI && n % 3) return PSX_ERR_ARG;
  if (value_precision != PSX_FP64 && value_precision != PSX_FP32_MIXED) return PSX_ERR_ARG;
  PcgWork w;
  int64_t need = 0;
  int rc = layout(n, precond, work, &w, &need);
  if (rc != PSX_OK) return rc;
  if (work_bytes < need) return PSX_ERR_ARG;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Status* st = static_cast<Status*>(status);
  const bool blk = precond == PSX_PRECOND_BJACOBI;
  const int id = precond == PSX_PRECOND_NONE;
#define PSX_RUN(VT, BLK, NOD) \
  run_pcg<VT, BLK, NOD>(n, indptr, indices, static_cast<const VT*>(values), b, x, rtol, atol, maxiter, w, st, s, id, \
                        host_checks)
  if (value_precision == PSX_FP64) {
    if (nodal) return blk ? PSX_RUN(double, true, true) : PSX_RUN(double, false, true);
    return blk ? PSX_RUN(double, true, false) : PSX_RUN(double, false, false);
  }
  if (nodal) return blk ? PSX_RUN(float, true, true) : PSX_RUN(float, false, true);
  return blk ? PSX_RUN(float, true, false) : PSX_RUN(float, false, false);
#undef PSX_RUN
}
}  // namespace

extern "C" int psx_pcg(int64_t n, const int32_t* indptr, const int32_t* indices, const void* values,
                       int value_precision, const double* b, double* x, double rtol, double atol, int32_t maxiter,
                       int precond, void* work, int64_t work_bytes, void* status, void* stream) {
  return pcg_entry(n, indptr, indices, values, value_precision, b, x, rtol, atol, maxiter, precond, work, work_bytes,
                   status, stream, true);
}

extern "C" int psx_pcg_coarse(int64_t n, const int32_t* indptr, const int32_t* indices, const void* values,
                              int value_precision, const double* b, double* x, double rtol, double atol,
                              int32_t maxiter, int precond, const psx_coarse_t* coarse, void* work,
                              int64_t work_bytes, void* status, void* stream, int host_checks) {
  using namespace psx;
  if (n <= 0 || !indptr || !indices || !values || !b || !x || !work || !status || maxiter < 0) return PSX_ERR_ARG;
  const bool nodal = (precond & PSX_PCG_NODAL) != 0;
  if ((precond & ~PSX_PCG_NODAL) != PSX_PRECOND_BJACOBI || n % 3) return PSX_ERR_ARG;
  if (!coarse_ok(coarse) || coarse->n_nodes * 3 != n) return coarse && coarse->nc > kCoarseMaxNc ? PSX_ERR_LIMIT : PSX_ERR_ARG;
  if (value_precision != PSX_FP64 && value_precision != PSX_FP32_MIXED) return PSX_ERR_ARG;
  PcgWork w;
  int64_t need = 0;
  int rc = layout(n, PSX_PRECOND_BJACOBI, work, &w, &need);
  if (rc != PSX_OK) return rc;
  if (work_bytes < need) return PSX_ERR_ARG;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Status* st = static_cast<Status*>(status);
  const bool hc = host_checks != 0;
  if (value_precision == PSX_FP64) {
    const double* v = static_cast<const double*>(values);
    return nodal ? run_pcg_coarse<double, true>(n, indptr, indices, v, b, x, rtol, atol, maxiter, w, *coarse, st, s, hc)
                 : run_pcg_coarse<double, false>(n, indptr, indices, v, b, x, rtol, atol, maxiter, w, *coarse, st, s, hc);
  }
  const float* v = static_cast<const float*>(values);
  return nodal ? run_pcg_coarse<float, true>(n, indptr, indices, v, b, x, rtol, atol, maxiter, w, *coarse, st, s, hc)
               : run_pcg_coarse<float, false>(n, indptr, indices, v, b, x, rtol, atol, maxiter, w, *coarse, st, s, hc);
}

extern "C" int psx_pcg_batched_work_bytes(int64_t n, int32_t n_seg, int64_t* bytes) {
  using namespace psx;
  if (n <= 0 || n % 3 || n_seg <= 0 || !bytes) return PSX_ERR_ARG;
  PcgWork w;
  int64_t vec = 0;
  layout(n, PSX_PRECOND_BJACOBI, nullptr, &w, &vec);
  *bytes = vec + (int64_t)up256(sizeof(SegScalars) * (size_t)n_seg);
  return PSX_OK;
}

extern "C" int psx_pcg_batched(int64_t n, const int32_t* indptr, const int32_t* indices, const void* values,
                               int value_precision, const double* b, double* x, double rtol, double atol,
                               int32_t maxiter, int precond, int32_t n_seg, const int64_t* seg_offsets,
                               const int32_t* node_seg, const psx_coarse_t* coarse, void* work, int64_t work_bytes,
                               void* status, int32_t* seg_iters, void* stream) {
  using namespace psx;
  if (n <= 0 || !indptr || !indices || !values || !b || !x || !work || !status || maxiter < 0 || n_seg <= 0 ||
      !seg_offsets || !node_seg)
    return PSX_ERR_ARG;
  const bool nodal = (precond & PSX_PCG_NODAL) != 0;
  if ((precond & ~PSX_PCG_NODAL) != PSX_PRECOND_BJACOBI || n % 3) return PSX_ERR_ARG;
  if (coarse && (!coarse_ok(coarse) || coarse->n_nodes * 3 != n))
    return coarse->nc > kCoarseMaxNc ? PSX_ERR_LIMIT : PSX_ERR_ARG;
  if (value_precision != PSX_FP64 && value_precision != PSX_FP32_MIXED) return PSX_ERR_ARG;
  int64_t need = 0;
  if (psx_pcg_batched_work_bytes(n, n_seg, &need) != PSX_OK || work_bytes < need) return PSX_ERR_ARG;
  PcgWork w;
  int64_t vec = 0;
  int rc = layout(n, PSX_PRECOND_BJACOBI, work, &w, &vec);
  if (rc != PSX_OK) return rc;
  BatchArgs ba{n_seg, seg_offsets, node_seg, reinterpret_cast<SegScalars*>(static_cast<char*>(work) + vec)};
  const psx_coarse_t c = coarse ? *coarse : psx_coarse_t{};
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Status* st = static_cast<Status*>(status);
#define PSX_RUN(VT, NOD, CO)                                                                                        \
  run_pcg_batched<VT, NOD, CO>(n, indptr, indices, static_cast<const VT*>(values), b, x, rtol, atol, maxiter, w, ba, \
                               c, st, seg_iters, s)
  if (value_precision == PSX_FP64) {
    if (nodal) return coarse ? PSX_RUN(double, true, true) : PSX_RUN(double, true, false);
    return coarse ? PSX_RUN(double, false, true) : PSX_RUN(double, false, false);
  }
  if (nodal) return coarse ? PSX_RUN(float, true, true) : PSX_RUN(float, true, false);
  return coarse ? PSX_RUN(float, false, true) : PSX_RUN(float, false, false);
#undef PSX_RUN
}

extern "C" int psx_coarse_probe(const psx_coarse_t* coarse, const int32_t* agg_color, int32_t color, int32_t mode,
                                double* v, void* stream) {
  using namespace psx;
  if (!coarse_ok(coarse) || !agg_color || !v || mode < 0 || mode > 5) return PSX_ERR_ARG;
  const int grid = (int)std::min<int64_t>(kGridMax, (coarse->n_nodes + kBlock - 1) / kBlock);
  coarse_probe_kernel<<<grid, kBlock, 0, static_cast<cudaStream_t>(stream)>>>(*coarse, agg_color, color, mode, v);
  PSX_CUDA_CHECK_LAUNCH();
  return PSX_OK;
}

extern "C" int psx_coarse_restrict(const psx_coarse_t* coarse, const double* w, double* out, void* stream) {
  using namespace psx;
  if (!coarse_ok(coarse) || !w || !out) return PSX_ERR_ARG;
  const int grid = (int)std::min<int64_t>(kGridMax, (coarse->n_agg + kBlock / 32 - 1) / (kBlock / 32));
  coarse_restrict_kernel<<<grid, kBlock, 0, static_cast<cudaStream_t>(stream)>>>(*coarse, w, out, nullptr);
  PSX_CUDA_CHECK_LAUNCH();
  return PSX_OK;
}

extern "C" int psx_pcg_enqueue(int64_t n, const int32_t* indptr, const int32_t* indices, const void* values,
                               int value_precision, const double* b, double* x, double rtol, double atol,
                               int32_t maxiter, int precond, void* work, int64_t work_bytes, void* status,
                               void* stream) {
  return pcg_entry(n, indptr, indices, values, value_precision, b, x, rtol, atol, maxiter, precond, work, work_bytes,
                   status, stream, false);
}

// ---------------------------------------------------------------------------------------
// Symmetric elimination of prescribed DOFs in a CSR matrix (in place): rows and columns
// of fixed DOFs are zeroed and their diagonal set to 1, which keeps the matrix symmetric
// positive definite and its pattern (and node alignment) unchanged.
namespace {
template <typename VT>
__global__ void csr_dirichlet_kernel(int64_t n, const int32_t* __restrict__ indptr,
                                     const int32_t* __restrict__ indices, VT* __restrict__ vals,
                                     const uint8_t* __restrict__ fixed) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
    const bool fr = fixed[r] != 0;
    for (int32_t j = indptr[r]; j < indptr[r + 1]; ++j) {
      const int32_t c = indices[j];
      if (fr)
        vals[j] = (c == r) ? (VT)1 : (VT)0;
      else if (fixed[c])
        vals[j] = (VT)0;
    }
  }
}
}  // namespace

extern "C" int psx_csr_dirichlet(int64_t n, const int32_t* indptr, const int32_t* indices, void* values,
                                 int value_precision, const uint8_t* fixed, void* stream) {
  if (n <= 0 || !indptr || !indices || !values || !fixed) return PSX_ERR_ARG;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int grid = (int)std::min<int64_t>(148 * 8, (n + 255) / 256);
  if (value_precision == PSX_FP64)
    csr_dirichlet_kernel<double><<<grid, 256, 0, s>>>(n, indptr, indices, static_cast<double*>(values), fixed);
  else if (value_precision == PSX_FP32_MIXED)
    csr_dirichlet_kernel<float><<<grid, 256, 0, s>>>(n, indptr, indices, static_cast<float*>(values), fixed);
  else
    return PSX_ERR_ARG;
  PSX_CUDA_CHECK_LAUNCH();
  return PSX_OK;
}

// ---------------------------------------------------------------------------------------
// y = alpha A x + beta y on a CSR matrix (8 lanes per row, fixed-order lane sums), the
// products M a and K_0 v of the dynamic residual.
namespace {
template <typename VT>
__global__ void __launch_bounds__(psx::kBlock) csr_spmv_kernel(int64_t n, const int32_t* __restrict__ indptr,
                                                                const int32_t* __restrict__ indices,
                                                                const VT* __restrict__ vals,
                                                                const double* __restrict__ x, double alpha,
                                                                double beta, double* __restrict__ y) {
  using namespace psx;
  const int lane8 = threadIdx.x & (kRowLanes - 1);
  const int64_t rows_per_pass = (int64_t)gridDim.x * (kBlock / kRowLanes);
  for (int64_t row0 = blockIdx.x * (int64_t)(kBlock / kRowLanes); row0 < n; row0 += rows_per_pass) {
    const int64_t row = row0 + threadIdx.x / kRowLanes;
    const double ax = spmv_row<VT>(n, row, lane8, indptr, indices, vals, x);
    if (row < n && lane8 == 0) y[row] = alpha * ax + (beta != 0.0 ? beta * y[row] : 0.0);
  }
}
}  // namespace

extern "C" int psx_csr_spmv(int64_t n, const int32_t* indptr, const int32_t* indices, const void* values,
                            int value_precision, const double* x, double alpha, double beta, double* y,
                            void* stream) {
  using namespace psx;
  if (n <= 0 || !indptr || !indices || !values || !x || !y) return PSX_ERR_ARG;
  if (value_precision != PSX_FP64 && value_precision != PSX_FP32_MIXED) return PSX_ERR_ARG;
  const int grid = (int)std::min<int64_t>(kGridMax, (n + kBlock / kRowLanes - 1) / (kBlock / kRowLanes));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (value_precision == PSX_FP64)
    csr_spmv_kernel<double><<<grid, kBlock, 0, s>>>(n, indptr, indices, static_cast<const double*>(values), x, alpha,
                                                    beta, y);
  else
    csr_spmv_kernel<float><<<grid, kBlock, 0, s>>>(n, indptr, indices, static_cast<const float*>(values), x, alpha,
                                                   beta, y);
  PSX_CUDA_CHECK_LAUNCH();
  return PSX_OK;
}

// ---------------------------------------------------------------------------------------
// Per-segment sums of squares (one block per segment, fixed reduction tree): the residual
// norms of the meshes of a batch, whose DOFs occupy contiguous ranges of one vector.
namespace {
__global__ void __launch_bounds__(psx::kBlock) segment_sumsq_kernel(int64_t n_seg, const int64_t* __restrict__ offsets,
                                                                     const double* __restrict__ x,
                                                                     double* __restrict__ out) {
  for (int64_t sgi = blockIdx.x; sgi < n_seg; sgi += gridDim.x) {
    const int64_t lo = offsets[sgi], hi = offsets[sgi + 1];
    double v[1] = {0.0};
    for (int64_t i = lo + threadIdx.x; i < hi; i += psx::kBlock) v[0] += x[i] * x[i];
    psx::block_sum<1>(v);
    if (threadIdx.x == 0) out[sgi] = v[0];
  }
}
}  // namespace

extern "C" int psx_segment_sumsq(int64_t n_seg, const int64_t* offsets, const double* x, double* out, void* stream) {
  if (n_seg <= 0 || !offsets || !x || !out) return PSX_ERR_ARG;
  const int grid = (int)std::min<int64_t>(n_seg, 148 * 8);
  segment_sumsq_kernel<<<grid, psx::kBlock, 0, static_cast<cudaStream_t>(stream)>>>(n_seg, offsets, x, out);
  PSX_CUDA_CHECK_LAUNCH();
  return PSX_OK;
}

// ---------------------------------------------------------------------------------------
// Allocation-free variant: psx_pcg_static.
//
// Some callers cannot hand this library a workspace.  A host code that owns all device
// memory through its own pool (a solver framework's arena, or PyTorch's caching
// allocator) cannot let a library call cudaMalloc behind its back: the allocation
// escapes the pool's accounting and implicitly synchronises the device.  A time-stepping
// loop that reserves its device memory up front may also forbid allocation mid-run.  For
// them the CG solve can run on scratch that is part of this library's image: a fixed
// array in device global memory, reserved on every GPU that loads the library until the
// process exits.
namespace {

constexpr size_t kStaticPcgBytes = size_t(32) << 20;  // 32 MiB of scratch per GPU
__device__ __align__(256) unsigned char g_pcg_scratch[kStaticPcgBytes];

constexpr int kMaxDevices = 64;
void* g_pcg_scratch_addr[kMaxDevices] = {};
std::mutex g_pcg_scratch_mu;

// Device address of the scratch array on the current device, looked up once per device
// with that device current (the host-side symbol is only a stand-in, not an address).
int static_scratch(void** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return PSX_ERR_CUDA;
  if (dev < 0 || dev >= kMaxDevices) return PSX_ERR_LIMIT;
  std::lock_guard<std::mutex> lock(g_pcg_scratch_mu);
  if (!g_pcg_scratch_addr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_pcg_scratch) != cudaSuccess || !p) return PSX_ERR_CUDA;
    g_pcg_scratch_addr[dev] = p;
  }
  *out = g_pcg_scratch_addr[dev];
  return PSX_OK;
}

}  // namespace

extern "C" size_t psx_pcg_static_max_bytes(void) { return kStaticPcgBytes; }

extern "C" int psx_pcg_static(int64_t n, const int32_t* indptr, const int32_t* indices, const void* values,
                              int value_precision, const double* b, double* x, double rtol, double atol,
                              int32_t maxiter, int precond, void* status, void* stream) {
  int64_t need = 0;
  int rc = psx_pcg_work_bytes(n, precond, &need);
  if (rc != PSX_OK) return rc;
  if (need > (int64_t)kStaticPcgBytes) return PSX_ERR_LIMIT;  // system too large for the fixed scratch
  void* scratch = nullptr;
  rc = static_scratch(&scratch);
  if (rc != PSX_OK) return rc;
  // psx_pcg clears the solver scalars and counters at the start of every call and
  // writes every vector before reading it, so the previous call's contents do not leak.
  return psx_pcg(n, indptr, indices, values, value_precision, b, x, rtol, atol, maxiter, precond, scratch,
                 (int64_t)kStaticPcgBytes, status, stream);
}
