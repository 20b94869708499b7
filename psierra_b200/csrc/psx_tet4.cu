// Tet4 Total-Lagrangian NeoHookean assembly kernels for sm_100a.
//
// Replaces the per-element Python loops of SolidDomain (psierra domain/solid.py:172-207,
// 230-274, 280-325) around Tet4TotalLagrangian.compute_nonlinear_force_and_tangent_stiffness
// (element/tet4_total_lagrangian.py:77-139) and the COO->CSR / np.add.at scatter
// (utility/assembly.py:37-108).
//
// Two phases per element chunk, fused into one launch per chunk:
//   A (element-centric): one thread per element evaluates the kinematics, the NeoHookean
//     stress and tangent, its 10 distinct 3x3 tangent blocks and its 4 nodal force
//     vectors, once, and writes them to an L2-resident ring of element records
//     (psx_gather.cuh).
//   B (owner-computes gather): one thread per node pair / node sums the records of the
//     elements that share it, in ascending element order, and writes each CSR value and
//     each f entry exactly once.
// Both phases run in one persistent launch that drains a task queue in mesh order, so
// the ring only holds the elements still awaited by some gather item.  No atomics touch f or K, so
// results are bitwise reproducible run to run.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "psx_common.cuh"
#include "psx_gather.cuh"
#include "psx_tet4_math.cuh"

namespace psx {
namespace {

constexpr int kThreads = 128;
constexpr int kModeDR = 16;       // internal: PSX_KV with the fused dynamic-relaxation epilogue
constexpr int kModeAdjoint = 64;  // internal: vector-Jacobian product of f_int
constexpr int kModeEff = 128;     // internal: c_t K_T + c_m M + c_0 K_0 (dynamic effective tangent)
#ifndef PSX_TET4_MIN_BLOCKS
#define PSX_TET4_MIN_BLOCKS 3
#endif
constexpr int kMinBlocks = PSX_TET4_MIN_BLOCKS;  // resident blocks per SM the register budget targets
// Register targets of the other instantiations (resident blocks per SM, which is also
// the default grid): the FP32 tangent without f, the FP64 tangent, the sweeps that build
// no tangent (f only, K.v, dynamic relaxation) and the adjoint.  Chosen by timing the
// 3.07M-element cube: more resident warps hide the element phase's latency, as long as
// the element tile fits the budget without spilling.
#ifndef PSX_TET4_TWO_PASS
#define PSX_TET4_TWO_PASS 1
#endif
#ifndef PSX_TET4_MIN_BLOCKS_K32
#define PSX_TET4_MIN_BLOCKS_K32 3
#endif
#ifndef PSX_TET4_MIN_BLOCKS_K64
#define PSX_TET4_MIN_BLOCKS_K64 2
#endif
#ifndef PSX_TET4_MIN_BLOCKS_NOK
#define PSX_TET4_MIN_BLOCKS_NOK 4
#endif
#ifndef PSX_TET4_MIN_BLOCKS_ADJ
#define PSX_TET4_MIN_BLOCKS_ADJ 2
#endif

struct Tet4Args {
  const int32_t* conn;
  const double* X;
  const double* U;
  const double* Vv;  // vector of the matrix-free product (PSX_KV) / cotangent (adjoint)
  double* dmu;       // adjoint: d(w.f)/d mu_e (E), or null
  double* dkappa;    // adjoint: d(w.f)/d kappa_e (E), or null
  const double* mu_e;
  const double* kappa_e;
  double mu0, kappa0, lam0;
  Status* st;
  // effective tangent (kModeEff): K_eff = c_t K_T + c_m M + c_0 K_0, M the consistent mass
  // of density rho, K_0 the small-strain stiffness (lam0, mu0, or per element
  // lambda = kappa_e - 2/3 mu_e, mu_e)
  double c_t, c_m, c_0, rho;
  // element records in the global ring (store_planes): the ring length (set by run_tet4)
  int64_t plane = 0;
};

// Phase A: one element -> its record.  tet4_total_lagrangian.py:77-139 (and, with
// PSX_LINEAR, tet4_base.py:129-136) in the closed form of psx_common.cuh.
// `krec` is global memory when KGLOBAL, else the shared-memory staging slot of the lane;
// `frec` is always global memory.
// 12 f / y doubles of an element: an L2-only store to the global ring, or plain stores to
// the shared-memory staging of the element tile.
template <bool FGLOBAL>
__device__ __forceinline__ void store_f12(double* __restrict__ frec, const double v[12], int64_t plane = 0) {
  if constexpr (FGLOBAL) {
    store_planes<double, 12>(frec, 0, v, plane);  // frec = ring + 2 * slot
  } else {
    double2* fq = reinterpret_cast<double2*>(frec);
#pragma unroll
    for (int i = 0; i < 6; ++i) fq[i] = make_double2(v[2 * i], v[2 * i + 1]);
  }
}

// A block of the element's record: planes of the global ring (KGLOBAL: krec = ring +
// W * slot), or the lane's shared-memory staging (krec = the staged record).
template <typename KT, bool KGLOBAL>
__device__ __forceinline__ void put_pair(KT* __restrict__ krec, int o, const KT b[9], bool swap, int64_t plane) {
  if constexpr (KGLOBAL) {
    KT v[12];
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int m = 0; m < 3; ++m) v[3 * k + m] = swap ? b[3 * m + k] : b[3 * k + m];
    v[9] = v[10] = v[11] = (KT)0;
    store_planes<KT, 12>(krec, o, v, plane);
  } else {
    store_pair_block<KT, false>(krec + o, b, swap);
  }
}
template <typename KT, bool KGLOBAL>
__device__ __forceinline__ void put_diag(KT* __restrict__ krec, int o, const KT d[6], int64_t plane) {
  if constexpr (KGLOBAL) {
    const KT v[8] = {d[0], d[1], d[2], d[3], d[4], d[5], (KT)0, (KT)0};
    store_planes<KT, 8>(krec, o, v, plane);
  } else {
    store_diag_block<KT, false>(krec + o, d);
  }
}

// Explicitly rounded operations in the tangent's type (dmul / fmul etc. of psx_common.cuh).
__device__ __forceinline__ double xmul(double a, double b) { return dmul(a, b); }
__device__ __forceinline__ float xmul(float a, float b) { return fmul(a, b); }
__device__ __forceinline__ double xadd(double a, double b) { return dadd(a, b); }
__device__ __forceinline__ float xadd(float a, float b) { return fadd(a, b); }
__device__ __forceinline__ double xfma(double a, double b, double c) { return dfma(a, b, c); }
__device__ __forceinline__ float xfma(float a, float b, float c) { return ffma(a, b, c); }
template <typename T>
__device__ __forceinline__ T xdot3(T a0, T b0, T a1, T b1, T a2, T b2) {
  return xfma(a0, b0, xfma(a1, b1, xmul(a2, b2)));
}

// `cn` = the element's connectivity (loaded by the caller, possibly ahead of time).
template <typename KT, int MODE, bool KGLOBAL = true, bool FGLOBAL = true>
__device__ __forceinline__ void tet4_element(const Tet4Args& A, int64_t e, const int4 cn, KT* __restrict__ krec,
                                             double* __restrict__ frec) {
  using L = RecLayout<4>;
  constexpr bool kAdj = (MODE & kModeAdjoint) != 0;
  constexpr bool kKV = (MODE & PSX_KV) != 0 || kAdj;
  constexpr bool kWantF = (MODE & PSX_WANT_F) != 0 && !kKV;
  constexpr bool kLinear = (MODE & PSX_LINEAR) != 0;
  constexpr bool kMass = (MODE & PSX_MASS) != 0;
  constexpr bool kWantK = ((MODE & PSX_WANT_K) != 0 || kLinear) && !kKV;
  double Xn[4][3];
  load_nodes(A.X, cn, Xn);
  // sweeps forming a tangent or K.v load the displacements with the coordinates (one
  // round trip to memory); the f-only sweep, with fewer registers in use, is faster
  // loading them after the geometry
  constexpr bool kEarlyU = !kMass && !kLinear && (kWantK || kKV);
  double Un[4][3];
  if constexpr (kEarlyU) load_nodes(A.U, cn, Un);
  Tet4Geom G;
  tet4_geometry(Xn, G);
  if (!(G.detD > 0.0)) flag_bad_element(A.st, e, true);
  if constexpr (kMass) {
    // tet4_base.py:138-151 with the volume of the mesh (|det| / 6, domain/solid.py:209-228)
    const KT mm = (KT)(A.lam0 * fabs(G.V) / 20.0);
    const KT off[9] = {mm, 0, 0, 0, mm, 0, 0, 0, mm};
    const KT d[6] = {(KT)2 * mm, 0, 0, (KT)2 * mm, 0, (KT)2 * mm};
#pragma unroll
    for (int slot = 0; slot < 6; ++slot) put_pair<KT, KGLOBAL>(krec, L::pair_off(slot), off, false, A.plane);
#pragma unroll
    for (int a = 0; a < 4; ++a) put_diag<KT, KGLOBAL>(krec, L::diag_off(a), d, A.plane);
    return;
  }
  KT p[4][3], q[4][3];
  TangentCoef<KT> tc;
  KT gk[4][3];
  // copies kept for the adjoint branch (dead code otherwise)
  double ps_F[3][3], ps_Finv[3][3], ps_P[3][3], ps_lnJ = 0.0, Un_[4][3], l_[3][3];
#pragma unroll
  for (int b = 0; b < 4; ++b)
#pragma unroll
    for (int k = 0; k < 3; ++k) gk[b][k] = (KT)G.g[b][k];
  if constexpr (kLinear) {
    // small-strain: p = q = g, K_ab = V [lam g_a g_b^T + mu g_b g_a^T + mu (g_a.g_b) I]
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
      for (int k = 0; k < 3; ++k) p[b][k] = q[b][k] = gk[b][k];
    tc.A = (KT)(G.V * A.lam0);
    tc.hb = (KT)(G.V * A.mu0);
    tc.c = (KT)0;
    tc.phi = (KT)(G.V * A.mu0);
  } else {
    const double mu = A.mu_e ? A.mu_e[e] : A.mu0;
    const double kappa = A.kappa_e ? A.kappa_e[e] : A.kappa0;
    double l[3][3];
    if constexpr (!kEarlyU) load_nodes(A.U, cn, Un);
    tet4_grad(Un, G, l);
    PointState ps;
    neohookean_point(l, mu, kappa, ps);
    if (G.detD > 0.0 && ps.Jm1 <= -1.0) flag_bad_element(A.st, e, false);
    if constexpr (kAdj) {
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          ps_F[i][j] = ps.F[i][j];
          ps_Finv[i][j] = ps.Finv[i][j];
          ps_P[i][j] = ps.P[i][j];
          l_[i][j] = l[i][j];
        }
      ps_lnJ = ps.lnJ;
#pragma unroll
      for (int b = 0; b < 4; ++b)
#pragma unroll
        for (int k = 0; k < 3; ++k) Un_[b][k] = Un[b][k];
    }
    if constexpr (kWantF) {
      double fr[12];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int i = 0; i < 3; ++i)
          fr[3 * a + i] = dmul(G.V, ddot3(ps.P[i][0], G.g[a][0], ps.P[i][1], G.g[a][1], ps.P[i][2], G.g[a][2]));
      store_f12<FGLOBAL>(frec, fr, A.plane);
    }
    if constexpr (kWantK || kKV) {
      tc = tangent_coef<KT>(ps, kappa, G.V);
      KT Fi[3][3], Fm[3][3];
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          Fi[i][j] = (KT)ps.Finv[i][j];
          Fm[i][j] = (KT)ps.F[i][j];
        }
#pragma unroll
      for (int b = 0; b < 4; ++b)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          p[b][k] = xdot3(Fi[0][k], gk[b][0], Fi[1][k], gk[b][1], Fi[2][k], gk[b][2]);
          q[b][k] = xdot3(Fm[k][0], gk[b][0], Fm[k][1], gk[b][1], Fm[k][2], gk[b][2]);
        }
    }
  }
  if constexpr (kKV) {
    // y_a = sum_b K_ab v_b = alpha p_a + Pv h_a + beta (c q_a) + phi (sum_b (g_a.g_b) v_b)
    // with alpha = sum_b w_b.v_b, beta = sum_b p_b.v_b, Pv = sum_b p_b v_b^T.
    // L2 loads: in the fused dynamic-relaxation step the vector is updated in place later
    // in the same launch (after every element reading a node has been evaluated).
    double Vn[4][3];
    {
      const int ids[4] = {cn.x, cn.y, cn.z, cn.w};
#pragma unroll
      for (int b = 0; b < 4; ++b)
#pragma unroll
        for (int k = 0; k < 3; ++k) Vn[b][k] = __ldcg(A.Vv + 3 * (int64_t)ids[b] + k);
    }
    KT vk[4][3];
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
      for (int k = 0; k < 3; ++k) vk[b][k] = (KT)Vn[b][k];
    KT alpha = 0, beta = 0, Pv[3][3], Gv[3][3];
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int m = 0; m < 3; ++m) Pv[k][m] = Gv[k][m] = (KT)0;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        alpha = xfma(xfma(tc.A, p[b][k], xmul(tc.c, q[b][k])), vk[b][k], alpha);
        beta = xfma(p[b][k], vk[b][k], beta);
#pragma unroll
        for (int m = 0; m < 3; ++m) {
          Pv[k][m] = xfma(p[b][k], vk[b][m], Pv[k][m]);
          Gv[k][m] = xfma(gk[b][k], vk[b][m], Gv[k][m]);
        }
      }
    }
    double yr[12];
    if constexpr (!kAdj) {
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          KT t = xfma(alpha, p[a][k], xmul(xmul(beta, tc.c), q[a][k]));
#pragma unroll
          for (int m = 0; m < 3; ++m)
            t = xadd(t, xfma(Pv[k][m], xmul(tc.hb, p[a][m]), xmul(xmul(tc.phi, gk[a][m]), Gv[m][k])));
          yr[3 * a + k] = (double)t;
        }
    } else {
      // Vector-Jacobian product of w.f_e with f_e,a = V P g_a (the adjoint of
      // tet4_total_lagrangian.py:136-137 w.r.t. X, mu, kappa).  L_w = sum_b w_b g_b^T,
      // VM = V dP/dF[L_w] = alpha F^-T + hb Pv F^-T + beta c F + phi Gv^T.
      double Fi[3][3], Fm[3][3], VM[3][3], Lw[3][3];
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          Fi[i][j] = (double)ps_Finv[i][j];
          Fm[i][j] = (double)ps_F[i][j];
          Lw[i][j] = 0.0;
        }
#pragma unroll
      for (int b = 0; b < 4; ++b)
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int j = 0; j < 3; ++j) Lw[i][j] += Vn[b][i] * G.g[b][j];
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int m = 0; m < 3; ++m) {
          // (F^-T)[k][m] = Finv[m][k]
          double t = (double)alpha * Fi[m][k] + (double)beta * (double)tc.c * Fm[k][m] + (double)tc.phi * (double)Gv[m][k];
#pragma unroll
          for (int j = 0; j < 3; ++j) t += (double)Pv[k][j] * (double)tc.hb * Fi[m][j];
          VM[k][m] = t;
        }
      // h_b = VM^T u_b + V P^T w_b  (vectors conjugate to dg_b)
      double h[4][3];
#pragma unroll
      for (int b = 0; b < 4; ++b)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          double t = 0.0;
#pragma unroll
          for (int i = 0; i < 3; ++i) t += VM[i][j] * Un_[b][i] + G.V * ps_P[i][j] * Vn[b][i];
          h[b][j] = t;
        }
      double PL = 0.0;
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) PL += ps_P[i][j] * Lw[i][j];
      // dL/dD = PL V G^T - G^T Hm G^T with G = D^-1 (rows g_1..g_3), Hm rows h_b - h_0
      double Gm[3][3], Hm[3][3], T1[3][3], Z[3][3];
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          Gm[r][j] = G.g[r + 1][j];
          Hm[r][j] = h[r + 1][j] - h[0][j];
        }
#pragma unroll
      for (int i = 0; i < 3; ++i)  // T1 = G^T Hm
#pragma unroll
        for (int j = 0; j < 3; ++j) T1[i][j] = Gm[0][i] * Hm[0][j] + Gm[1][i] * Hm[1][j] + Gm[2][i] * Hm[2][j];
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
          Z[i][j] = PL * G.V * Gm[j][i] - (T1[i][0] * Gm[j][0] + T1[i][1] * Gm[j][1] + T1[i][2] * Gm[j][2]);
      // D[i][j] = X_{j+1}[i] - X_0[i]
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        yr[i] = -(Z[i][0] + Z[i][1] + Z[i][2]);
#pragma unroll
        for (int j = 0; j < 3; ++j) yr[3 * (j + 1) + i] = Z[i][j];
      }
      // parameter gradients: dP/dmu = 2 J^-2/3 F^-T dev E, dP/dkappa = ln J F^-T
      if (A.dmu || A.dkappa) {
        double E[3][3], trE = 0.0;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int j = 0; j < 3; ++j) {
            const double ltl = l_[0][i] * l_[0][j] + l_[1][i] * l_[1][j] + l_[2][i] * l_[2][j];
            E[i][j] = 0.5 * (l_[i][j] + l_[j][i] + ltl);
          }
        trE = E[0][0] + E[1][1] + E[2][2];
        const double jm23 = exp((-2.0 / 3.0) * ps_lnJ);
        double FTL = 0.0, FDL = 0.0;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int j = 0; j < 3; ++j) {
            FTL += Fi[j][i] * Lw[i][j];
            double fd = 0.0;  // (F^-T dev E)[i][j]
#pragma unroll
            for (int k = 0; k < 3; ++k) fd += Fi[k][i] * (E[k][j] - (k == j ? trE / 3.0 : 0.0));
            FDL += fd * Lw[i][j];
          }
        if (A.dmu) A.dmu[e] = G.V * 2.0 * jm23 * FDL;
        if (A.dkappa) A.dkappa[e] = G.V * ps_lnJ * FTL;
      }
    }
    store_f12<FGLOBAL>(frec, yr);
  }
  if constexpr (kWantK) {
    // K_ab[k][m] = p_a,k w_b,m + p_b,k h_a,m + y_a,k p_b,m + s_ab d_km
    constexpr bool kEff = (MODE & kModeEff) != 0;
    KT e_lam = 0, e_mu = 0, e_mass = 0;  // effective tangent: K_0 and mass coefficients
    if constexpr (kEff) {
      const KT ct = (KT)A.c_t;
      tc.A *= ct;
      tc.hb *= ct;
      tc.c *= ct;
      tc.phi *= ct;
      const double mu_k = A.mu_e ? A.mu_e[e] : A.mu0;
      const double lam_k = A.mu_e ? dfma(-2.0 / 3.0, A.mu_e[e], A.kappa_e[e]) : A.lam0;
      e_lam = (KT)(A.c_0 * G.V * lam_k);
      e_mu = (KT)(A.c_0 * G.V * mu_k);
      e_mass = (KT)(A.c_m * A.rho * fabs(G.V) * (1.0 / 20.0));  // element/tet4_base.py:138-151
    }
    // FP32 tangent staged in shared memory: the element's factors go through its own
    // staging slot (and are read back after a compiler barrier), so none of the FP64
    // kinematic and constitutive state is live while the ten blocks are formed; this
    // keeps the register count of the fused f + K tile low enough for 3 blocks per SM
    constexpr bool kTwoPass = PSX_TET4_TWO_PASS && !KGLOBAL && sizeof(KT) == 4 && !kLinear && !kMass;
    if constexpr (kTwoPass) {
      // 44 floats as 11 16-byte accesses: with the 108-float slot stride the 8 lanes of
      // each access phase fall on disjoint banks (scalar accesses put 4 lanes on a bank)
      float v[44];
#pragma unroll
      for (int b = 0; b < 4; ++b)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          v[3 * b + k] = (float)p[b][k];
          v[12 + 3 * b + k] = (float)q[b][k];
          v[24 + 3 * b + k] = (float)gk[b][k];
        }
      v[36] = (float)tc.A;
      v[37] = (float)tc.hb;
      v[38] = (float)tc.c;
      v[39] = (float)tc.phi;
      v[40] = (float)e_lam;
      v[41] = (float)e_mu;
      v[42] = (float)e_mass;
      v[43] = 0.f;
      float4* fs = reinterpret_cast<float4*>(krec);
#pragma unroll
      for (int i = 0; i < 11; ++i) fs[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
      asm volatile("" ::: "memory");
#pragma unroll
      for (int i = 0; i < 11; ++i) {
        const float4 t = fs[i];
        v[4 * i] = t.x;
        v[4 * i + 1] = t.y;
        v[4 * i + 2] = t.z;
        v[4 * i + 3] = t.w;
      }
#pragma unroll
      for (int b = 0; b < 4; ++b)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          p[b][k] = (KT)v[3 * b + k];
          q[b][k] = (KT)v[12 + 3 * b + k];
          gk[b][k] = (KT)v[24 + 3 * b + k];
        }
      tc.A = (KT)v[36];
      tc.hb = (KT)v[37];
      tc.c = (KT)v[38];
      tc.phi = (KT)v[39];
      e_lam = (KT)v[40];
      e_mu = (KT)v[41];
      e_mass = (KT)v[42];
    }
    KT w[4][3], h[4][3], y[4][3];
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        w[b][k] = xfma(tc.A, p[b][k], xmul(tc.c, q[b][k]));
        h[b][k] = xmul(tc.hb, p[b][k]);
        y[b][k] = xmul(tc.c, q[b][k]);
      }
    const int gid[4] = {cn.x, cn.y, cn.z, cn.w};
    int slot = 0;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
#pragma unroll
      for (int b = a; b < 4; ++b) {
        const KT gg = xdot3(gk[a][0], gk[b][0], gk[a][1], gk[b][1], gk[a][2], gk[b][2]);
        KT s = xmul(tc.phi, gg);
        if constexpr (kEff) s = xadd(s, xfma(e_mu, gg, xmul(e_mass, a == b ? (KT)2 : (KT)1)));
        KT v[9];
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
          for (int m = 0; m < 3; ++m) {
            const KT last = k == m ? xfma(y[a][k], p[b][m], s) : xmul(y[a][k], p[b][m]);
            v[3 * k + m] = xfma(p[a][k], w[b][m], xfma(p[b][k], h[a][m], last));
            if constexpr (kEff)
              v[3 * k + m] = xadd(v[3 * k + m], xfma(xmul(e_lam, gk[a][k]), gk[b][m], xmul(xmul(e_mu, gk[b][k]), gk[a][m])));
          }
        if (b == a) {
          const KT d[6] = {v[0], v[1], v[2], v[4], v[5], v[8]};
          put_diag<KT, KGLOBAL>(krec, L::diag_off(a), d, A.plane);
        } else {
          put_pair<KT, KGLOBAL>(krec, L::pair_off(slot), v, gid[a] > gid[b], A.plane);
          ++slot;
        }
      }
    }
  }
}

// Persistent assembly kernel: each warp repeatedly claims the next task of the queue
// (psx_task_fill).  Element tiles publish their granule's completion count; gather
// tiles wait for the element granules they read; element tiles wait until the gather
// tiles still reading the ring slots they overwrite are done.  Every wait is on tasks
// that earlier warps have already claimed, so the queue always drains.  There are no
// block-wide barriers: warps of a block progress independently.
//
// Tile records (FP32 tangent, and every sweep without a tangent): the 32 elements of a
// warp's tile stage their blocks and f triples in shared memory; the warp then sums the
// blocks its elements share (psx_tile_plan_fill: local pairs / nodes by descending
// contribution count, contributions in element order) and writes one record per distinct pair and
// node, with consecutive lanes on consecutive records.  The FP64 tangent writes one
// record per element straight to the ring.
constexpr int kStageStride = RecLayout<4>::kK + 4;  // floats per staged element record (bank spread)
constexpr int kFStride = 14;                        // doubles per staged f triple set (bank spread)

// Largest per-tile meta block the shared-memory list area holds (tile = 32).
constexpr int kMetaBytes = 656;

template <typename KT, int MODE>
struct Tet4Smem {
  static constexpr bool kKV = (MODE & (PSX_KV | kModeAdjoint)) != 0;
  static constexpr bool kWantK = (MODE & (PSX_WANT_K | PSX_LINEAR | PSX_MASS)) != 0 && !kKV;
  static constexpr bool kWantF = (MODE & PSX_WANT_F) != 0 || kKV;
  static constexpr bool kTiles = sizeof(KT) == 4 || !kWantK;
  static constexpr int kKFloats = kTiles && kWantK ? 32 * kStageStride : 0;  // per warp
  static constexpr int kFDoubles = kTiles && kWantF ? 32 * kFStride : 0;    // per warp
  static constexpr int kMeta = kTiles ? kMetaBytes : 0;                       // per warp
  static constexpr size_t kWarpBytes = sizeof(float) * kKFloats + sizeof(double) * kFDoubles + kMeta;
};

// Asynchronous 16-byte global -> shared copies (no registers held while in flight).
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Start copying tile t's meta block into the warp's list area: the whole block for a
// sweep with a tangent, the count bytes and node lists (its first meta_node_bytes) for
// the sweeps without one (f-only 20.5 -> 8.5 bytes of lists per element).
template <bool WANT_K>
__device__ __forceinline__ void tile_meta_prefetch(const GatherArgs& g, int64_t t, unsigned char* lst) {
  const int lane = threadIdx.x & 31;
  const uint4* src = reinterpret_cast<const uint4*>(g.tile_meta + t * g.meta_stride);
  const int chunks = (WANT_K ? g.meta_stride : g.meta_node_bytes) / 16;
  for (int c = lane; c < chunks; c += 32) cp_async16(lst + 16 * c, src + c);
}

// Sum the staged element blocks of tile `t` into its tile record (one warp), with the
// tile's lists in shared memory (`lst`, tile_meta_prefetch).  The record is stored in
// planes (gather_args): pair values 0-3, 4-7 and 8, diagonal xx xy xz yy and yz zz, and
// f x, y, z, each plane contiguous over the tile's pairs or nodes, so that every store
// of the warp writes whole sectors.
template <bool WANT_K, bool WANT_F>
__device__ __forceinline__ void tile_reduce(const GatherArgs& g, int64_t t, const unsigned char* __restrict__ lst,
                                            const float* __restrict__ kst, const double* __restrict__ fst,
                                            float* __restrict__ krec, double* __restrict__ frec) {
  using L = RecLayout<4>;
  const int lane = threadIdx.x & 31;
  const int64_t slot = t & g.ring_tile_mask;
  float* kbase = krec + slot * g.tile_k;
  if constexpr (WANT_K) {
    const int np = lst[0];
    const unsigned char* off = lst + g.off_p;
    const unsigned char* src = lst + g.src_p;
    float4* p0 = reinterpret_cast<float4*>(kbase);
    float4* p1 = reinterpret_cast<float4*>(kbase + 4 * g.cap_p4);
    float* p2 = kbase + 8 * g.cap_p4;
    for (int lp = lane; lp < np; lp += 32) {
      const int a0 = off[lp], a1 = off[lp + 1];
      float4 s0 = make_float4(0.f, 0.f, 0.f, 0.f), s1 = s0;
      float s2 = 0.f;
      #pragma unroll 1
      for (int q = a0; q < a1; ++q) {
        const int c = src[q];
        const float* b = kst + (c >> 3) * kStageStride + L::pair_off(c & 7);
        const float4 x = reinterpret_cast<const float4*>(b)[0], y = reinterpret_cast<const float4*>(b)[1];
        s0.x += x.x; s0.y += x.y; s0.z += x.z; s0.w += x.w;
        s1.x += y.x; s1.y += y.y; s1.z += y.z; s1.w += y.w;
        s2 += b[8];
      }
      st_ring(p0 + lp, s0);
      st_ring(p1 + lp, s1);
      st_ring(p2 + lp, s2);
    }
  }
  const int nn = lst[1];
  const unsigned char* off = lst + g.off_n;
  const unsigned char* src = lst + g.src_n;
  float4* d0p = reinterpret_cast<float4*>(kbase + 9 * g.cap_p4);
  float2* d1p = reinterpret_cast<float2*>(kbase + 9 * g.cap_p4 + 4 * g.cap_n4);
  double* fb = frec + slot * 3 * g.cap_n4;
  for (int ln = lane; ln < nn; ln += 32) {
    const int a0 = off[ln], a1 = off[ln + 1];
    float4 d0 = make_float4(0.f, 0.f, 0.f, 0.f);
    float2 d1 = make_float2(0.f, 0.f);
    double f0 = 0.0, f1 = 0.0, f2 = 0.0;
    #pragma unroll 1
    for (int q = a0; q < a1; ++q) {
      const int c = src[q];
      const int el = c >> 2, a = c & 3;
      if constexpr (WANT_K) {
        const float4* b = reinterpret_cast<const float4*>(kst + el * kStageStride + L::diag_off(a));
        const float4 x = b[0];
        const float2 y = reinterpret_cast<const float2*>(b + 1)[0];
        d0.x += x.x; d0.y += x.y; d0.z += x.z; d0.w += x.w;
        d1.x += y.x; d1.y += y.y;
      }
      if constexpr (WANT_F) {
        const double* fp = fst + el * kFStride + 3 * a;
        f0 += fp[0];
        f1 += fp[1];
        f2 += fp[2];
      }
    }
    if constexpr (WANT_K) {
      st_ring(d0p + ln, d0);
      st_ring(d1p + ln, d1);
    }
    if constexpr (WANT_F) {
      st_ring(fb + ln, f0);
      st_ring(fb + g.cap_n4 + ln, f1);
      st_ring(fb + 2 * g.cap_n4 + ln, f2);
    }
  }
}

template <typename KT, int MODE>
constexpr int min_blocks() {
  return (MODE & kModeAdjoint) != 0 ? PSX_TET4_MIN_BLOCKS_ADJ
         : (MODE & (PSX_WANT_K | PSX_LINEAR | PSX_MASS)) == 0 || (MODE & PSX_KV) != 0
             ? PSX_TET4_MIN_BLOCKS_NOK
             : (sizeof(KT) == 8 ? PSX_TET4_MIN_BLOCKS_K64 : ((MODE & PSX_WANT_F) ? kMinBlocks : PSX_TET4_MIN_BLOCKS_K32));
}

template <typename KT, int MODE>
__global__ void __launch_bounds__(kThreads, min_blocks<KT, MODE>())
tet4_persistent_kernel(Tet4Args A, GatherArgs g, QueueArgs Q, KT* __restrict__ krec, double* __restrict__ frec,
                       KT* __restrict__ k_out, double* __restrict__ f_out, DRArgs dr) {
  using L = RecLayout<4>;
  using S = Tet4Smem<KT, MODE>;
  constexpr bool kDR = (MODE & kModeDR) != 0;
  const int lane = threadIdx.x & 31;
  extern __shared__ __align__(16) unsigned char s_stage[];  // kThreads/32 warps x S::kWarpBytes
  unsigned char* my_stage = s_stage + (threadIdx.x >> 5) * S::kWarpBytes;
  float* kst = reinterpret_cast<float*>(my_stage);
  double* fst = reinterpret_cast<double*>(my_stage + sizeof(float) * S::kKFloats);
  unsigned char* lst = my_stage + sizeof(float) * S::kKFloats + sizeof(double) * S::kFDoubles;
  auto element_tile = [&](const int4& task) {
    if constexpr (S::kTiles) {
      // a tile is `g.tile` consecutive elements starting at a multiple of g.tile; its
      // lists arrive in shared memory while the elements are evaluated
      const int64_t t = task.z / g.tile;
      tile_meta_prefetch<S::kWantK>(g, t, lst);
      const int64_t e = task.z + (int64_t)lane;
      if (e < task.w)
        tet4_element<KT, MODE, false, false>(A, e, __ldg(reinterpret_cast<const int4*>(A.conn) + e),
                                             reinterpret_cast<KT*>(kst + lane * kStageStride), fst + kFStride * lane);
      cp_async_wait_all();
      __syncwarp();
      tile_reduce<S::kWantK, S::kWantF>(g, t, lst, kst, fst, reinterpret_cast<float*>(krec), frec);
      __syncwarp();  // the staging and the lists are reused by the warp's next tile
    } else {
      for (int64_t e = task.z + (int64_t)lane; e < task.w; e += 32) {
        const int64_t slot = e & g.ring_mask;
        tet4_element<KT, MODE>(A, e, __ldg(reinterpret_cast<const int4*>(A.conn) + e),
                               krec + slot * (16 / (int64_t)sizeof(KT)), frec + slot * 2);  // planar records
      }
    }
  };
  drain_queue<KT, 4, S::kWantK, S::kWantF, kDR, S::kTiles>(g, Q, A.st, krec, frec, k_out, f_out, dr, element_tile);
}

// Warp-specialised FP32 tangent sweep: one block of 16 warps per SM.  Warpgroups 0-1
// evaluate element tiles and stage them in shared memory (setmaxnreg raises them to
// kSplitElemRegs registers), warpgroups 2-3 run the gathers (lowered to
// kSplitGatherRegs).  The gathers' dependent loads then hide behind more warps than the
// element phase's register need allows in the mixed kernel.  What the gather warps
// release must cover what the element warps take, so the launch must give each thread
// exactly kSplitLaunchRegs registers (run_tet4_split checks the compiled kernel).
//
// Measured on the 3.07M-element cube (f+K):
// * roles: 12 element + 4 gather warps 1.2-1.4 ms and 4 + 12 1.6 ms (either role
//   starves), 20 or 24 warps per block (fewer registers per role, spills) 0.98-1.09 ms,
//   8 + 8 with 160-184 element registers within 2-4 % of each other;
// * contributions in flight per gather lane: 2 pair blocks (0.672 ms against 0.694 with
//   1, and 0.687 with 2 pair and 2 node blocks, with the planar tile records);
// * the sweeps without a tangent (f, K.v, DR step) stay on the mixed kernel: their FP64
//   element phase is the bottleneck and their node gathers are light, so giving half
//   the warps to gathers doubled their time (K.v 0.30 -> 0.58 ms with 8 + 8 warps).
#ifndef PSX_SPLIT_PAIR_BATCH_FK
#define PSX_SPLIT_PAIR_BATCH_FK 2
#endif
#ifndef PSX_SPLIT_PAIR_BATCH_K
#define PSX_SPLIT_PAIR_BATCH_K 2
#endif
#ifndef PSX_SPLIT_NODE_BATCH
#define PSX_SPLIT_NODE_BATCH 1
#endif
// 176 element / 80 gather registers: 160 / 96 measured 0.645-0.652 ms against
// 0.616-0.621 on the 80^3 cube (f+K)
#ifndef PSX_SPLIT_ELEM_REGS
#define PSX_SPLIT_ELEM_REGS 176
#endif
#ifndef PSX_SPLIT_ELEM_WARPS
#define PSX_SPLIT_ELEM_WARPS 8
#endif
#ifndef PSX_SPLIT_THREADS
#define PSX_SPLIT_THREADS 512
#endif
constexpr int kSplitThreads = PSX_SPLIT_THREADS;
constexpr int kSplitElemWarps = PSX_SPLIT_ELEM_WARPS;
constexpr int kSplitLaunchRegs = 65536 / kSplitThreads / 8 * 8;  // what __launch_bounds__(threads, 1) allows
constexpr int kSplitElemRegs = PSX_SPLIT_ELEM_REGS;
// what the element warps take beyond the launch allocation, the gather warps give up
constexpr int kSplitGatherRegs =
    ((kSplitThreads / 32) * kSplitLaunchRegs - kSplitElemWarps * kSplitElemRegs) / (kSplitThreads / 32 - kSplitElemWarps) /
    8 * 8;
static_assert(kSplitThreads % 128 == 0 && kSplitThreads * kSplitLaunchRegs <= 65536, "one block per SM, whole warpgroups");
static_assert(kSplitElemWarps * kSplitElemRegs + (kSplitThreads / 32 - kSplitElemWarps) * kSplitGatherRegs <=
                  (kSplitThreads / 32) * kSplitLaunchRegs,
              "the register split must fit the launch allocation");
static_assert(kSplitElemWarps % 4 == 0 && kSplitElemWarps < kSplitThreads / 32, "roles are whole warpgroups");
static_assert(kSplitElemRegs % 8 == 0 && kSplitElemRegs <= 256 && kSplitGatherRegs >= 24, "setmaxnreg range");

template <typename KT, int MODE>
__global__ void __launch_bounds__(kSplitThreads, 1)
tet4_split_kernel(Tet4Args A, GatherArgs g, QueueArgs Q, const int4* __restrict__ gtasks, int32_t n_gtasks,
                  KT* __restrict__ krec, double* __restrict__ frec, KT* __restrict__ k_out, double* __restrict__ f_out) {
  using S = Tet4Smem<KT, MODE>;
  static_assert(S::kTiles && S::kWantK && sizeof(KT) == 4, "the split kernel runs FP32 tangent sweeps");
  extern __shared__ __align__(16) unsigned char s_stage[];  // kSplitElemWarps x S::kWarpBytes
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  int32_t* ecnt = Q.counters;
  int32_t* gcnt = Q.counters + 1 + 2 * Q.n_granules;
  if (warp < kSplitElemWarps) {
    asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;\n" ::"n"(kSplitElemRegs));
    unsigned char* my_stage = s_stage + warp * S::kWarpBytes;
    float* kst = reinterpret_cast<float*>(my_stage);
    double* fst = reinterpret_cast<double*>(my_stage + sizeof(float) * S::kKFloats);
    unsigned char* lst = my_stage + sizeof(float) * S::kKFloats + sizeof(double) * S::kFDoubles;
    drain_elements(Q, reinterpret_cast<const int4*>(A.conn), ecnt, A.st,
                   [&](const int4& task, const int4 cn, auto&& publish_previous) {
      const int64_t t = task.z / g.tile;
      tile_meta_prefetch<S::kWantK>(g, t, lst);
      const int64_t e = task.z + (int64_t)lane;
      if (e < task.w)
        tet4_element<KT, MODE, false, false>(A, e, cn, reinterpret_cast<KT*>(kst + lane * kStageStride),
                                             fst + kFStride * lane);
      cp_async_wait_all();
      __syncwarp();
      publish_previous();
      tile_reduce<S::kWantK, S::kWantF>(g, t, lst, kst, fst, reinterpret_cast<float*>(krec), frec);
      __syncwarp();
    });
  } else {
    asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;\n" ::"n"(kSplitGatherRegs));
    constexpr int kPairBatch = S::kWantF ? PSX_SPLIT_PAIR_BATCH_FK : PSX_SPLIT_PAIR_BATCH_K;
    drain_gathers<KT, 4, S::kWantK, S::kWantF, kPairBatch, PSX_SPLIT_NODE_BATCH>(
        g, Q, gtasks, n_gtasks, gcnt, A.st, krec, frec, k_out, f_out);
  }
}

// The split kernel is usable when its compiled register count is the one its
// setmaxnreg split is computed for (checked once per process: the count is a property
// of the compiled kernel).
template <typename KT, int MODE>
bool split_usable() {
  static int s_regs = -1;
  if (s_regs < 0) {
    cudaFuncAttributes fa{};
    if (cudaFuncGetAttributes(&fa, tet4_split_kernel<KT, MODE>) != cudaSuccess) return false;
    s_regs = fa.numRegs;
  }
  return s_regs == kSplitLaunchRegs;
}

__global__ void tet4_dets_kernel(const int32_t* __restrict__ conn, const double* __restrict__ X,
                                 const double* __restrict__ U, int64_t e, double* out2) {
  const int4 cn = reinterpret_cast<const int4*>(conn)[e];
  double Xn[4][3];
  load_nodes(X, cn, Xn);
  Tet4Geom G;
  tet4_geometry(Xn, G);
  out2[0] = G.detD;
  if (U) {
    double Un[4][3], l[3][3];
    load_nodes(U, cn, Un);
    tet4_grad(Un, G, l);
    double F[3][3];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) F[i][j] = (i == j ? 1.0 : 0.0) + l[i][j];
    out2[1] = det3(F);
  } else {
    out2[1] = 1.0;
  }
}

template <typename KT, int MODE>
int run_tet4(const psx_plan_t* P, const Tet4Args& A, const WorkLayout& W, KT* k_out, double* f_out,
             cudaStream_t stream, const DRArgs& dr = DRArgs{}) {
  constexpr bool kWantK =
      (MODE & (PSX_WANT_K | PSX_LINEAR | PSX_MASS)) != 0 && (MODE & (PSX_KV | kModeAdjoint)) == 0;
  const GatherArgs g = gather_args(P, W.ring_elems);
  const QueueArgs Q = queue_args(P, W, kWantK);
  using S = Tet4Smem<KT, MODE>;
  // the kernel's record format (tile or element records) must be the one the workspace
  // was laid out for
  if (W.tiles != S::kTiles) return PSX_ERR_ARG;
  if (S::kTiles && (P->tile > 32 || g.tile_k % 4 || g.meta_stride > kMetaBytes)) return PSX_ERR_ARG;
  if (cudaMemsetAsync(W.counters, 0, W.counter_bytes, stream) != cudaSuccess) return PSX_ERR_CUDA;
  const size_t smem = (kThreads / 32) * S::kWarpBytes;
  static unsigned long long s_smem_set = 0;
  if (smem > 0 && set_dynamic_smem_once(tet4_persistent_kernel<KT, MODE>, (int)smem, &s_smem_set) != cudaSuccess)
    return PSX_ERR_CUDA;
  // one block per SM per register-target block, unless the plan overrides it
  int grid = W.grid;
  if (P->blocks_per_sm <= 0) {
    const int64_t ntask = Q.n_tasks;
    const int64_t want = (int64_t)device_sm_count() * min_blocks<KT, MODE>();
    grid = (int)(want < ntask ? want : ntask);
    if (grid <= 0) grid = 1;
  }
  Tet4Args Ap = A;
  Ap.plane = W.ring_elems;  // element records are stored in planes of the ring (store_planes)
  tet4_persistent_kernel<KT, MODE><<<grid, kThreads, smem, stream>>>(Ap, g, Q, static_cast<KT*>(W.krec), W.frec,
                                                                    k_out, f_out, dr);
  PSX_CUDA_CHECK_LAUNCH();
  return PSX_OK;
}

template <typename KT, int MODE>
int run_tet4_split(const psx_plan_t* P, const Tet4Args& A, const WorkLayout& W, KT* k_out, double* f_out,
                   cudaStream_t stream) {
  using S = Tet4Smem<KT, MODE>;
  const GatherArgs g = gather_args(P, W.ring_elems);
  const QueueArgs Q = queue_args(P, W, true);
  if (!W.tiles || !S::kTiles || P->tile > 32 || g.tile_k % 4 || g.meta_stride > kMetaBytes) return PSX_ERR_ARG;
  if (!P->gtasks_k || P->n_gtasks_k <= 0 || P->n_gtasks_k > 0x7fffffff) return PSX_ERR_ARG;
  if (cudaMemsetAsync(W.counters, 0, W.counter_bytes, stream) != cudaSuccess) return PSX_ERR_CUDA;
  const size_t smem = kSplitElemWarps * S::kWarpBytes;
  static unsigned long long s_smem_set = 0;
  if (set_dynamic_smem_once(tet4_split_kernel<KT, MODE>, (int)smem, &s_smem_set) != cudaSuccess) return PSX_ERR_CUDA;
  const int grid = device_sm_count();  // one block (the whole register file) per SM
  if (grid <= 0) return PSX_ERR_CUDA;
  tet4_split_kernel<KT, MODE><<<grid, kSplitThreads, smem, stream>>>(
      A, g, Q, reinterpret_cast<const int4*>(P->gtasks_k), (int32_t)P->n_gtasks_k, static_cast<KT*>(W.krec), W.frec,
      k_out, f_out);
  PSX_CUDA_CHECK_LAUNCH();
  return PSX_OK;
}

// FP32 tangent sweeps take the warp-specialised kernel when the plan carries the gather
// task list and the kernel's register split is valid; otherwise the mixed kernel.
template <int MODE>
int run_tet4_k32(const psx_plan_t* P, const Tet4Args& A, const WorkLayout& W, float* k_out, double* f_out,
                 cudaStream_t stream) {
  if (P->gtasks_k && P->n_gtasks_k > 0 && W.tiles && split_usable<float, MODE>())
    return run_tet4_split<float, MODE>(P, A, W, k_out, f_out, stream);
  return run_tet4<float, MODE>(P, A, W, k_out, f_out, stream);
}

}  // namespace
}  // namespace psx

extern "C" size_t psx_status_bytes(void) { return sizeof(psx::Status); }

extern "C" int psx_tet4_split_ready(void) {
  return psx::split_usable<float, PSX_WANT_F | PSX_WANT_K>() && psx::split_usable<float, PSX_WANT_K>() ? 1 : 0;
}

extern "C" int psx_work_bytes(const psx_plan_t* plan, int precision, int64_t* ring_elems, int64_t* bytes) {
  // one workspace serves both task queues: the larger of their layouts
  psx::WorkLayout Wk, Wf;
  int rc = psx::work_layout(plan, precision, nullptr, &Wk, 3, true);
  if (rc != PSX_OK) return rc;
  rc = psx::work_layout(plan, precision, nullptr, &Wf, 3, false);
  if (rc != PSX_OK) return rc;
  if (!ring_elems || !bytes) return PSX_ERR_ARG;
  *ring_elems = Wk.ring_elems > Wf.ring_elems ? Wk.ring_elems : Wf.ring_elems;
  *bytes = Wk.total_bytes > Wf.total_bytes ? Wk.total_bytes : Wf.total_bytes;
  return PSX_OK;
}

extern "C" int psx_tet4_assemble(const psx_plan_t* plan, const double* X, const double* u, const double* mu_e,
                                 const double* kappa_e, double mu, double kappa, double lam, int mode,
                                 int precision, double* f_out, void* k_out, void* work, int64_t work_bytes,
                                 void* status, void* stream) {
  using namespace psx;
  if (!plan || plan->npe != 4 || !X || !status || !work) return PSX_ERR_ARG;
  const bool wantF = (mode & PSX_WANT_F) != 0, wantK = (mode & PSX_WANT_K) != 0,
             mass = (mode & PSX_MASS) != 0, linear = (mode & PSX_LINEAR) != 0 || mass;
  if ((mode & PSX_LINEAR) && mass) return PSX_ERR_ARG;
  if (linear && (wantF || wantK || !k_out)) return PSX_ERR_ARG;
  if (!linear && (!(wantF || wantK) || !u)) return PSX_ERR_ARG;
  if (wantF && !f_out) return PSX_ERR_ARG;
  if (wantK && !k_out) return PSX_ERR_ARG;
  WorkLayout W;
  int rc = work_layout(plan, precision, work, &W, kMinBlocks, wantK || linear);
  if (rc != PSX_OK) return rc;
  if (work_bytes < W.total_bytes) return PSX_ERR_ARG;
  Tet4Args A{plan->conn, X, u, nullptr, nullptr, nullptr, mu_e, kappa_e, mu, kappa, lam, static_cast<Status*>(status)};
  cudaStream_t s = static_cast<cudaStream_t>(stream);
#define PSX_T4(KT, M) run_tet4<KT, M>(plan, A, W, static_cast<KT*>(k_out), f_out, s)
  if (mass) return precision == PSX_FP64 ? PSX_T4(double, PSX_MASS) : PSX_T4(float, PSX_MASS);
  if (linear) return precision == PSX_FP64 ? PSX_T4(double, PSX_LINEAR) : PSX_T4(float, PSX_LINEAR);
  if (wantF && wantK)
    return precision == PSX_FP64 ? PSX_T4(double, PSX_WANT_F | PSX_WANT_K)
                                 : run_tet4_k32<PSX_WANT_F | PSX_WANT_K>(plan, A, W, static_cast<float*>(k_out),
                                                                         f_out, s);
  if (wantK)
    return precision == PSX_FP64 ? PSX_T4(double, PSX_WANT_K)
                                 : run_tet4_k32<PSX_WANT_K>(plan, A, W, static_cast<float*>(k_out), f_out, s);
  return PSX_T4(double, PSX_WANT_F);
#undef PSX_T4
}

extern "C" int psx_tet4_assemble_effective(const psx_plan_t* plan, const double* X, const double* u,
                                           const double* mu_e, const double* kappa_e, double mu, double kappa,
                                           double lam, double rho, double c_t, double c_m, double c_0, int mode,
                                           int precision, double* f_out, void* k_out, void* work, int64_t work_bytes,
                                           void* status, void* stream) {
  using namespace psx;
  if (!plan || plan->npe != 4 || !X || !u || !status || !work || !k_out) return PSX_ERR_ARG;
  if ((mode & PSX_WANT_K) == 0 || (mode & ~(PSX_WANT_F | PSX_WANT_K))) return PSX_ERR_ARG;
  if ((mode & PSX_WANT_F) && !f_out) return PSX_ERR_ARG;
  if ((mu_e == nullptr) != (kappa_e == nullptr)) return PSX_ERR_ARG;
  WorkLayout W;
  int rc = work_layout(plan, precision, work, &W, kMinBlocks, true);
  if (rc != PSX_OK) return rc;
  if (work_bytes < W.total_bytes) return PSX_ERR_ARG;
  Tet4Args A{plan->conn, X, u, nullptr, nullptr, nullptr, mu_e, kappa_e, mu, kappa, lam, static_cast<Status*>(status),
             c_t, c_m, c_0, rho};
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  constexpr int kFK = PSX_WANT_F | PSX_WANT_K | kModeEff, kK = PSX_WANT_K | kModeEff;
  // the FP32 effective tangent takes the warp-specialised kernel like K_T itself (the
  // element math is explicitly rounded, so both kernels give the same bits)
  if (mode & PSX_WANT_F)
    return precision == PSX_FP64 ? run_tet4<double, kFK>(plan, A, W, static_cast<double*>(k_out), f_out, s)
                                 : run_tet4_k32<kFK>(plan, A, W, static_cast<float*>(k_out), f_out, s);
  return precision == PSX_FP64 ? run_tet4<double, kK>(plan, A, W, static_cast<double*>(k_out), nullptr, s)
                               : run_tet4_k32<kK>(plan, A, W, static_cast<float*>(k_out), nullptr, s);
}

extern "C" int psx_tet4_kv(const psx_plan_t* plan, const double* X, const double* u, const double* mu_e,
                           const double* kappa_e, double mu, double kappa, int precision, const double* v,
                           double* y_out, void* work, int64_t work_bytes, void* status, void* stream) {
  using namespace psx;
  if (!plan || plan->npe != 4 || !X || !u || !v || !y_out || !status || !work) return PSX_ERR_ARG;
  WorkLayout W;
  int rc = work_layout(plan, precision, work, &W, kMinBlocks, false);
  if (rc != PSX_OK) return rc;
  if (work_bytes < W.total_bytes) return PSX_ERR_ARG;
  Tet4Args A{plan->conn, X, u, v, nullptr, nullptr, mu_e, kappa_e, mu, kappa, 0.0, static_cast<Status*>(status)};
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  return precision == PSX_FP64 ? run_tet4<double, PSX_KV>(plan, A, W, nullptr, y_out, s)
                               : run_tet4<float, PSX_KV>(plan, A, W, nullptr, y_out, s);
}

extern "C" int psx_tet4_dr_step(const psx_plan_t* plan, const double* X, const double* u, const double* mu_e,
                                const double* kappa_e, double mu, double kappa, int precision, const double* b,
                                const double* minv, double c1, double c2, double dt, double* x, double* vel,
                                double* r_out, void* work, int64_t work_bytes, void* status, void* stream) {
  using namespace psx;
  if (!plan || plan->npe != 4 || !X || !u || !b || !minv || !x || !vel || !status || !work) return PSX_ERR_ARG;
  WorkLayout W;
  int rc = work_layout(plan, precision, work, &W, kMinBlocks, false);
  if (rc != PSX_OK) return rc;
  if (work_bytes < W.total_bytes) return PSX_ERR_ARG;
  Tet4Args A{plan->conn, X, u, x, nullptr, nullptr, mu_e, kappa_e, mu, kappa, 0.0, static_cast<Status*>(status)};
  DRArgs dr{b, minv, c1, c2, dt, x, vel};
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  return precision == PSX_FP64 ? run_tet4<double, PSX_KV | kModeDR>(plan, A, W, nullptr, r_out, s, dr)
                               : run_tet4<float, PSX_KV | kModeDR>(plan, A, W, nullptr, r_out, s, dr);
}

extern "C" int psx_tet4_adjoint(const psx_plan_t* plan, const double* X, const double* u, const double* mu_e,
                                const double* kappa_e, double mu, double kappa, const double* w, double* gX_out,
                                double* gmu_out, double* gkappa_out, void* work, int64_t work_bytes, void* status,
                                void* stream) {
  using namespace psx;
  if (!plan || plan->npe != 4 || !X || !u || !w || !gX_out || !status || !work) return PSX_ERR_ARG;
  WorkLayout W;
  int rc = work_layout(plan, PSX_FP64, work, &W, kMinBlocks, false);
  if (rc != PSX_OK) return rc;
  if (work_bytes < W.total_bytes) return PSX_ERR_ARG;
  Tet4Args A{plan->conn, X, u, w, gmu_out, gkappa_out, mu_e, kappa_e, mu, kappa, 0.0, static_cast<Status*>(status)};
  return run_tet4<double, kModeAdjoint>(plan, A, W, nullptr, gX_out, static_cast<cudaStream_t>(stream));
}

extern "C" int psx_tet4_element_dets(const int32_t* conn, const double* X, const double* u, int64_t e,
                                     double* out2, void* stream) {
  if (!conn || !X || !out2 || e < 0) return PSX_ERR_ARG;
  psx::tet4_dets_kernel<<<1, 1, 0, static_cast<cudaStream_t>(stream)>>>(conn, X, u, e, out2);
  PSX_CUDA_CHECK_LAUNCH();
  return PSX_OK;
}
