// Shared device code for the Tet4/Tet10 Total-Lagrangian NeoHookean kernels.
//
// Element math follows pSierra's Tet4/Tet10 TL elements and NeoHookean material
// (psierra element/tet4_total_lagrangian.py:77-139, element/tet10_total_lagrangian.py:63-136,
// material/neohookean.py:55-122) in a closed, symmetry-exploiting form:
//
//   l  = sum_b u_b g_b^T          (displacement gradient, g_b = grad N_b)
//   F  = I + l,  J - 1 = tr l + ((tr l)^2 - tr l^2)/2 + det l   (no cancellation at small l)
//   ln J = log1p(J - 1),  phi = mu J^(-2/3),  beta = kappa ln J
//   S  = C^-1 (2 phi dev E + beta I),  E = (l + l^T + l^T l)/2     (== the reference's
//        phi (I - I1/3 C^-1) + beta C^-1, without its O(mu) cancellation)
//   f_a = V F S g_a
//   K_ab = V [ A p_a p_b^T + hb p_b p_a^T + c (p_a q_b^T + q_a p_b^T) + phi (g_a . g_b) I ]
//        with p_a = F^-T g_a, q_a = F g_a, A = kappa + 2/9 phi I1, hb = phi I1/3 - beta,
//        c = -2/3 phi.
//
// K_ab equals B_a^T C_voigt B_b V + G_a^T (I (x) S) G_b V of the reference: the
// C^-1 (x) C^-1, the symmetrised C^-1 product and the C^-1 (x) I terms of the 4th-order
// tangent contract with B = sym(F^T grad N) to the three outer products, and the
// p_a.p_b parts of the symmetrised term and of the geometric term cancel exactly.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "psierra_b200.h"

namespace psx {

struct Mat3 {
  double m[3][3];
};

// Explicitly rounded arithmetic for the element math.  Every multiply, add and fused
// multiply-add of the force and tangent is written out, so the compiler cannot fuse or
// reorder them differently in different kernels: the warp-specialised kernel, the mixed
// kernel and the effective-tangent kernel then compute the same bits for the same
// element (a schedule change never changes a result).
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dfma(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float ffma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
// a b - c d with c d rounded once
__device__ __forceinline__ double dmm(double a, double b, double c, double d) { return dfma(a, b, -dmul(c, d)); }
// a0 b0 + a1 b1 + a2 b2, accumulated from the last term
__device__ __forceinline__ double ddot3(double a0, double b0, double a1, double b1, double a2, double b2) {
  return dfma(a0, b0, dfma(a1, b1, dmul(a2, b2)));
}
__device__ __forceinline__ float fdot3(float a0, float b0, float a1, float b1, float a2, float b2) {
  return ffma(a0, b0, ffma(a1, b1, fmul(a2, b2)));
}

__device__ __forceinline__ double det3(const double a[3][3]) {
  return ddot3(a[0][0], dmm(a[1][1], a[2][2], a[1][2], a[2][1]), a[0][1], dmm(a[1][2], a[2][0], a[1][0], a[2][2]),
               a[0][2], dmm(a[1][0], a[2][1], a[1][1], a[2][0]));
}

// Inverse through the adjugate; returns the determinant.
__device__ __forceinline__ double inv3(const double a[3][3], double r[3][3]) {
  const double c00 = dmm(a[1][1], a[2][2], a[1][2], a[2][1]);
  const double c01 = dmm(a[0][2], a[2][1], a[0][1], a[2][2]);
  const double c02 = dmm(a[0][1], a[1][2], a[0][2], a[1][1]);
  const double c10 = dmm(a[1][2], a[2][0], a[1][0], a[2][2]);
  const double c11 = dmm(a[0][0], a[2][2], a[0][2], a[2][0]);
  const double c12 = dmm(a[0][2], a[1][0], a[0][0], a[1][2]);
  const double c20 = dmm(a[1][0], a[2][1], a[1][1], a[2][0]);
  const double c21 = dmm(a[0][1], a[2][0], a[0][0], a[2][1]);
  const double c22 = dmm(a[0][0], a[1][1], a[0][1], a[1][0]);
  const double det = ddot3(a[0][0], c00, a[0][1], c10, a[0][2], c20);
  const double id = 1.0 / det;
  r[0][0] = dmul(c00, id); r[0][1] = dmul(c01, id); r[0][2] = dmul(c02, id);
  r[1][0] = dmul(c10, id); r[1][1] = dmul(c11, id); r[1][2] = dmul(c12, id);
  r[2][0] = dmul(c20, id); r[2][1] = dmul(c21, id); r[2][2] = dmul(c22, id);
  return det;
}

// Kinematic + constitutive state of one integration point, everything in FP64.
struct PointState {
  double F[3][3];     // deformation gradient
  double Finv[3][3];  // F^-1
  double P[3][3];     // first Piola-Kirchhoff stress F S
  double Jm1;         // J - 1 (compensated)
  double lnJ;         // ln J
  double phi;         // mu J^(-2/3)
  double beta;        // kappa ln J
  double I1;          // tr C
};

// Constitutive update from the displacement gradient l (3x3, FP64).
// neohookean.py:74-92 restated without cancellation (see the header comment).
__device__ __forceinline__ void neohookean_point(const double l[3][3], double mu, double kappa,
                                                 PointState& s) {
  const double trl = dadd(dadd(l[0][0], l[1][1]), l[2][2]);
  double trl2 = dmul(l[0][0], l[0][0]);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int k = 0; k < 3; ++k)
      if (i + k > 0) trl2 = dfma(l[i][k], l[k][i], trl2);
  s.Jm1 = dadd(dadd(trl, dmul(0.5, dfma(trl, trl, -trl2))), det3(l));
  const double lnJ = log1p(s.Jm1);
  s.lnJ = lnJ;
  s.phi = dmul(mu, exp(dmul(-2.0 / 3.0, lnJ)));
  s.beta = dmul(kappa, lnJ);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) s.F[i][j] = i == j ? dadd(1.0, l[i][j]) : l[i][j];
  inv3(s.F, s.Finv);
  // Green-Lagrange strain E = (l + l^T + l^T l) / 2 (symmetric: six entries formed)
  double E[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = i; j < 3; ++j) {
      const double ltl = ddot3(l[0][i], l[0][j], l[1][i], l[1][j], l[2][i], l[2][j]);
      E[i][j] = dmul(0.5, dadd(dadd(l[i][j], l[j][i]), ltl));
      E[j][i] = E[i][j];
    }
  const double trE = dadd(dadd(E[0][0], E[1][1]), E[2][2]);
  s.I1 = dfma(2.0, trE, 3.0);
  // T = 2 phi dev E + beta I (symmetric)
  double T[3][3];
  const double tw = dmul(2.0, s.phi), dia = dfma(-tw, trE / 3.0, s.beta);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = i; j < 3; ++j) {
      T[i][j] = i == j ? dfma(tw, E[i][j], dia) : dmul(tw, E[i][j]);
      T[j][i] = T[i][j];
    }
  // S = C^-1 T, so P = F S = F F^-1 F^-T T = F^-T T: the first Piola stress without
  // forming C^-1 or S
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j)
      s.P[i][j] = ddot3(s.Finv[0][i], T[0][j], s.Finv[1][i], T[1][j], s.Finv[2][i], T[2][j]);
}

// Tangent coefficients with the integration weight folded in.
template <typename T>
struct TangentCoef {
  T A, hb, c, phi;
};

template <typename T>
__device__ __forceinline__ TangentCoef<T> tangent_coef(const PointState& s, double kappa, double w) {
  TangentCoef<T> t;
  t.A = (T)dmul(w, dfma(dmul(2.0 / 9.0, s.phi), s.I1, kappa));
  t.hb = (T)dmul(w, dsub(dmul(s.phi, s.I1) / 3.0, s.beta));
  t.c = (T)dmul(w, dmul(-2.0 / 3.0, s.phi));
  t.phi = (T)dmul(w, s.phi);
  return t;
}

// Stores of records into the ring that the gathers read back (element and tile records,
// their f triples), with an L2 evict_last policy: the ring stays resident while the CSR
// values, stored with the streaming hint, pass through L2.  Measured against plain .cg
// stores: Tet4 FP64 f+K on the 3.07M-element cube 1.564 -> 1.544 ms, Tet10 on the
// 162,000-element cube 0.662 -> 0.657 ms (FP32-mixed) and 1.024 -> 1.018 ms (FP64).
__device__ __forceinline__ unsigned long long l2_keep_policy() {
  unsigned long long p;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ void st_ring(float4* q, float4 v) {
  asm volatile("st.global.L2::cache_hint.v4.f32 [%0], {%1, %2, %3, %4}, %5;" ::"l"(q), "f"(v.x), "f"(v.y), "f"(v.z),
               "f"(v.w), "l"(l2_keep_policy())
               : "memory");
}
__device__ __forceinline__ void st_ring(float2* q, float2 v) {
  asm volatile("st.global.L2::cache_hint.v2.f32 [%0], {%1, %2}, %3;" ::"l"(q), "f"(v.x), "f"(v.y), "l"(l2_keep_policy())
               : "memory");
}
__device__ __forceinline__ void st_ring(double2* q, double2 v) {
  asm volatile("st.global.L2::cache_hint.v2.f64 [%0], {%1, %2}, %3;" ::"l"(q), "d"(v.x), "d"(v.y), "l"(l2_keep_policy())
               : "memory");
}
__device__ __forceinline__ void st_ring(float* q, float v) {
  asm volatile("st.global.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(q), "f"(v), "l"(l2_keep_policy()) : "memory");
}
__device__ __forceinline__ void st_ring(double* q, double v) {
  asm volatile("st.global.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(q), "d"(v), "l"(l2_keep_policy()) : "memory");
}

// Three consecutive CSR values at p (aligned to the value size) in two streaming stores:
// the two-value half that is aligned to twice the value size and the remaining value,
// chosen by predicates so that the lanes of a warp do not diverge.  Each pair block then
// costs 12 store instructions instead of 18, and fewer partial L2 sector writes.
__device__ __forceinline__ void store3(float* p, float a, float b, float c) {
  const bool al = (reinterpret_cast<uintptr_t>(p) & 7) == 0;
  float2* pv = reinterpret_cast<float2*>(al ? p : p + 1);
  __stcs(pv, al ? make_float2(a, b) : make_float2(b, c));
  __stcs(al ? p + 2 : p, al ? c : a);
}

__device__ __forceinline__ void store3(double* p, double a, double b, double c) {
  const bool al = (reinterpret_cast<uintptr_t>(p) & 15) == 0;
  __stcs(reinterpret_cast<double2*>(al ? p : p + 1), al ? make_double2(a, b) : make_double2(b, c));
  __stcs(al ? p + 2 : p, al ? c : a);
}

// Add (a, b, c) to three consecutive doubles at p (8-byte aligned), with the same
// vector + scalar split for the loads and the stores.
__device__ __forceinline__ void add3(double* p, double a, double b, double c) {
  const bool al = (reinterpret_cast<uintptr_t>(p) & 15) == 0;
  double2* pv = reinterpret_cast<double2*>(al ? p : p + 1);
  double* ps = al ? p + 2 : p;
  double2 v = *pv;
  double w = *ps;
  v.x += al ? a : b;
  v.y += al ? b : c;
  w += al ? c : a;
  *pv = v;
  *ps = w;
}

// Status words written by every element kernel (device side).  Counters are
// reset with a plain memset; `first_bad_key` stores INT32_MAX - e so that an
// atomicMax picks the lowest element index and a zeroed word means "none".
struct Status {
  int32_t n_inverted;     // elements with det F <= 0
  int32_t n_bad_volume;   // elements with reference det <= 0
  int32_t first_bad_key;  // INT32_MAX - (lowest bad element index), 0 if none
  int32_t n_not_finite;   // reserved for solver status
  int32_t iters;          // solver iterations (PCG)
  int32_t flags;          // solver flags
  double value;           // solver residual or auxiliary value
};

__device__ __forceinline__ void flag_bad_element(Status* st, int64_t e, bool volume) {
  if (volume)
    atomicAdd(&st->n_bad_volume, 1);
  else
    atomicAdd(&st->n_inverted, 1);
  atomicMax(&st->first_bad_key, (int32_t)(0x7fffffff - (int32_t)e));
}

// Raise a kernel's dynamic shared-memory limit once per device, so that later launches
// (including launches captured into a CUDA graph) make no attribute call.
template <typename K>
inline cudaError_t set_dynamic_smem_once(K* kernel, int bytes, unsigned long long* done_mask) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned long long bit = 1ull << (dev & 63);
  if (__atomic_load_n(done_mask, __ATOMIC_ACQUIRE) & bit) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) __atomic_fetch_or(done_mask, bit, __ATOMIC_RELEASE);
  return e;
}

}  // namespace psx

#define PSX_CUDA_CHECK_LAUNCH()                      \
  do {                                               \
    cudaError_t _e = cudaGetLastError();             \
    if (_e != cudaSuccess) return PSX_ERR_CUDA;      \
  } while (0)
