// Tet10 Total-Lagrangian NeoHookean assembly for sm_100a.
//
// Replaces the element loops of SolidDomain (psierra domain/solid.py:172-207, 230-325)
// around Tet10TotalLagrangian.compute_nonlinear_force_and_tangent_stiffness
// (element/tet10_total_lagrangian.py:63-136; shape gradients element/tet10_base.py:118-179,
// VTK edge order 4:(0,1) 5:(1,2) 6:(2,0) 7:(0,3) 8:(1,3) 9:(2,3); 4-point rule
// element/quadrature.py:36-49 with weight 1/24) and the COO->CSR / np.add.at scatter.
//
// Element tiles of up to 8 elements are evaluated by one warp in two phases:
//   1. lane 4*le + q handles element le of the tile at quadrature point q: Jacobian
//      J = X^T dN, det J, H = dN J^-1, the displacement gradient, the NeoHookean point
//      (psx_common.cuh), the nodal force contributions (reduced over the 4 q-lanes of
//      the element in a fixed tree) and, per node, p = F^-T H_a, q = F H_a, H_a into
//      shared memory with the weighted tangent coefficients;
//   2. the warp spreads the 8 x 55 3x3 blocks (45 node pairs + 10 diagonals) over its
//      lanes; each sums its block over the 4 quadrature points with the closed form of
//      psx_common.cuh and writes it into the element's record.
// The records are then gathered by the shared owner-computes queue (psx_gather.cuh).
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "psx_common.cuh"
#include "psx_gather.cuh"

namespace psx {
namespace {

constexpr int kThreads10 = 128;
constexpr int kTile10 = 8;  // elements per warp task (one per 4 lanes)
using L10 = RecLayout<10>;

// local node pairs (a < b) in slot order, then the 10 diagonals
struct PairTable {
  int8_t a[55], b[55];
};
__constant__ PairTable c_pairs = {
    {0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, 1, 1, 1, 2, 2, 2, 2, 2, 2, 2, 3, 3, 3, 3, 3, 3, 4, 4, 4, 4, 4, 5, 5, 5, 5,
     6, 6, 6, 7, 7, 8, 0, 1, 2, 3, 4, 5, 6, 7, 8, 9},
    {1, 2, 3, 4, 5, 6, 7, 8, 9, 2, 3, 4, 5, 6, 7, 8, 9, 3, 4, 5, 6, 7, 8, 9, 4, 5, 6, 7, 8, 9, 5, 6, 7, 8, 9, 6, 7, 8, 9,
     7, 8, 9, 8, 9, 9, 0, 1, 2, 3, 4, 5, 6, 7, 8, 9}};

// Consistent mass of the 10-node tetrahedron with straight edges: M_ab = rho V m_ab / 2520
// times the 3x3 identity, m_ab the exact integrals of N_a N_b over the reference element
// (VTK node order; element/tet10_base.py:11-27, 344-372).
__constant__ int16_t c_mass10[10][10] = {
    {36, 6, 6, 6, -24, -36, -24, -24, -36, -36},   {6, 36, 6, 6, -24, -24, -36, -36, -24, -36},
    {6, 6, 36, 6, -36, -24, -24, -36, -36, -24},   {6, 6, 6, 36, -36, -36, -36, -24, -24, -24},
    {-24, -24, -36, -36, 192, 96, 96, 96, 96, 48}, {-36, -24, -24, -36, 96, 192, 96, 48, 96, 96},
    {-24, -36, -24, -36, 96, 96, 192, 96, 48, 96}, {-24, -36, -36, -24, 96, 48, 96, 192, 96, 96},
    {-36, -24, -36, -24, 96, 96, 48, 96, 192, 96}, {-36, -36, -24, -24, 48, 96, 96, 96, 96, 192}};

// Barycentric coordinates (L1, L2, L3) of the 4-point rule: a = (5 - sqrt 5)/20,
// b = (5 + 3 sqrt 5)/20.
__device__ __forceinline__ void qp_coords(int q, double& L1, double& L2, double& L3) {
  const double a = 0.13819660112501051517954131656344, b = 0.58541019662496845446137605030969;
  L1 = q == 1 ? b : a;
  L2 = q == 2 ? b : a;
  L3 = q == 3 ? b : a;
}

// dN_a / d(xi, eta, zeta) at (L1, L2, L3); tet10_base.py:137-177.
__device__ __forceinline__ void shape_grad(int a, double L1, double L2, double L3, double d[3]) {
  const double L0 = 1.0 - L1 - L2 - L3;
  switch (a) {
    case 0: d[0] = d[1] = d[2] = -(4.0 * L0 - 1.0); break;
    case 1: d[0] = 4.0 * L1 - 1.0; d[1] = 0.0; d[2] = 0.0; break;
    case 2: d[0] = 0.0; d[1] = 4.0 * L2 - 1.0; d[2] = 0.0; break;
    case 3: d[0] = 0.0; d[1] = 0.0; d[2] = 4.0 * L3 - 1.0; break;
    case 4: d[0] = 4.0 * (L0 - L1); d[1] = -4.0 * L1; d[2] = -4.0 * L1; break;
    case 5: d[0] = 4.0 * L2; d[1] = 4.0 * L1; d[2] = 0.0; break;
    case 6: d[0] = -4.0 * L2; d[1] = 4.0 * (L0 - L2); d[2] = -4.0 * L2; break;
    case 7: d[0] = -4.0 * L3; d[1] = -4.0 * L3; d[2] = 4.0 * (L0 - L3); break;
    case 8: d[0] = 4.0 * L3; d[1] = 0.0; d[2] = 4.0 * L1; break;
    default: d[0] = 0.0; d[1] = 4.0 * L3; d[2] = 4.0 * L2; break;
  }
}

struct Tet10Args {
  const int32_t* conn;
  const double* X;
  const double* U;
  const double* mu_e;
  const double* kappa_e;
  double mu0, kappa0, lam0;
  Status* st;
};

// Shared-memory scratch of one warp: per (element, qp, node) p, q, H and per (element,
// qp) the weighted tangent coefficients.
template <typename KT>
struct Tet10Smem {
  KT p[kTile10][4][10][3];
  KT q[kTile10][4][10][3];
  KT h[kTile10][4][10][3];
  KT c[kTile10][4][4];  // A, hb, c, phi (times w det J)
};

template <typename KT, int MODE>
__device__ __forceinline__ void tet10_tile(const Tet10Args& A, const int4& task, int64_t ring_mask,
                                           KT* __restrict__ krec, double* __restrict__ frec, Tet10Smem<KT>& sm) {
  constexpr bool kLinear = (MODE & PSX_LINEAR) != 0;
  constexpr bool kWantF = (MODE & PSX_WANT_F) != 0 && !kLinear;
  constexpr bool kWantK = (MODE & PSX_WANT_K) != 0 || kLinear;
  const int lane = threadIdx.x & 31;
  if constexpr ((MODE & PSX_MASS) != 0) {
    // consistent mass (density in lam0) with the element volume of the mesh, |det| / 6 of
    // the corner tetrahedron (domain/solid.py:209-228): one 3x3 block per lane
    const int n = (int)(task.w - task.z);
    for (int t = lane; t < n * 55; t += 32) {
      const int me = t / 55, slot = t - me * 55;
      const int a = c_pairs.a[slot], b = c_pairs.b[slot];
      const int64_t em = task.z + me;
      double Xc[4][3];
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const double* x = A.X + 3 * (int64_t)__ldg(A.conn + 10 * em + c);
#pragma unroll
        for (int i = 0; i < 3; ++i) Xc[c][i] = __ldg(x + i);
      }
      double D[3][3];
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) D[i][j] = Xc[j + 1][i] - Xc[0][i];
      const double V = fabs(det3(D)) / 6.0;
      const KT m = (KT)(A.lam0 * V * (double)c_mass10[a][b] / 2520.0);
      KT* rec = krec + (em & ring_mask) * L10::kK;
      if (slot < 45) {
        const KT blk[9] = {m, (KT)0, (KT)0, (KT)0, m, (KT)0, (KT)0, (KT)0, m};
        store_pair_block<KT>(rec + L10::pair_off(slot), blk, false);
      } else {
        const KT dg[6] = {m, (KT)0, (KT)0, m, (KT)0, m};
        store_diag_block<KT>(rec + L10::diag_off(slot - 45), dg);
      }
    }
    return;
  }
  const int le = lane >> 2, q = lane & 3;
  const int64_t e = task.z + (int64_t)le;
  const bool active = e < task.w;
  // ---- phase 1: one (element, quadrature point) per lane
  double L1, L2, L3;
  qp_coords(q, L1, L2, L3);
  int32_t nid[10];
  if (active) {
    const int2* c2 = reinterpret_cast<const int2*>(A.conn + 10 * e);  // 40-byte rows are 8-byte aligned
#pragma unroll
    for (int i = 0; i < 5; ++i) {
      const int2 t = __ldg(c2 + i);
      nid[2 * i] = t.x;
      nid[2 * i + 1] = t.y;
    }
  } else {
#pragma unroll
    for (int i = 0; i < 10; ++i) nid[i] = 0;
  }
  double Jm[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
  for (int a = 0; a < 10; ++a) {
    double d[3];
    shape_grad(a, L1, L2, L3, d);
    const double* x = A.X + 3 * (int64_t)nid[a];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const double xi = active ? __ldg(x + i) : (i == (a % 3) ? 1.0 : 0.0);
#pragma unroll
      for (int j = 0; j < 3; ++j) Jm[i][j] += xi * d[j];
    }
  }
  double Ji[3][3];
  const double detJ = inv3(Jm, Ji);
  if (active && !(detJ > 0.0)) flag_bad_element(A.st, e, true);
  const double w = detJ / 24.0;
  double mu = A.mu0, kappa = A.kappa0;
  if (active && A.mu_e) mu = A.mu_e[e];
  if (active && A.kappa_e) kappa = A.kappa_e[e];
  PointState ps;
  TangentCoef<KT> tc;
  if constexpr (kLinear) {
    tc.A = (KT)(w * A.lam0);
    tc.hb = (KT)(w * A.mu0);
    tc.c = (KT)0;
    tc.phi = (KT)(w * A.mu0);
  } else {
    double l[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    double u0[3] = {0, 0, 0};
    if (active) {
      const double* up = A.U + 3 * (int64_t)nid[0];
      u0[0] = __ldg(up);
      u0[1] = __ldg(up + 1);
      u0[2] = __ldg(up + 2);
    }
#pragma unroll
    for (int a = 1; a < 10; ++a) {
      double d[3], H[3];
      shape_grad(a, L1, L2, L3, d);
#pragma unroll
      for (int j = 0; j < 3; ++j) H[j] = d[0] * Ji[0][j] + d[1] * Ji[1][j] + d[2] * Ji[2][j];
      const double* up = A.U + 3 * (int64_t)nid[a];
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        const double du = active ? __ldg(up + i) - u0[i] : 0.0;
#pragma unroll
        for (int j = 0; j < 3; ++j) l[i][j] += du * H[j];
      }
    }
    neohookean_point(l, mu, kappa, ps);
    if (active && detJ > 0.0 && ps.Jm1 <= -1.0) flag_bad_element(A.st, e, false);
    tc = tangent_coef<KT>(ps, kappa, w);
  }
  KT Fi[3][3], Fm[3][3];
  if constexpr (!kLinear) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        Fi[i][j] = (KT)ps.Finv[i][j];
        Fm[i][j] = (KT)ps.F[i][j];
      }
  }
#pragma unroll
  for (int a = 0; a < 10; ++a) {
    double d[3], H[3];
    shape_grad(a, L1, L2, L3, d);
#pragma unroll
    for (int j = 0; j < 3; ++j) H[j] = d[0] * Ji[0][j] + d[1] * Ji[1][j] + d[2] * Ji[2][j];
    if constexpr (kWantF) {
      // f_a += w P H_a, summed over the element's 4 q-lanes in a fixed tree
      double fa[3];
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        double v = active ? w * (ps.P[i][0] * H[0] + ps.P[i][1] * H[1] + ps.P[i][2] * H[2]) : 0.0;
        v += __shfl_xor_sync(0xffffffffu, v, 1);
        v += __shfl_xor_sync(0xffffffffu, v, 2);
        fa[i] = v;
      }
      if (active && q == 0) {
        double* fr = frec + (e & ring_mask) * L10::kF + 3 * a;
        st_ring(fr, fa[0]);
        st_ring(fr + 1, fa[1]);
        st_ring(fr + 2, fa[2]);
      }
    }
    if constexpr (kWantK) {
      const KT Hk[3] = {(KT)H[0], (KT)H[1], (KT)H[2]};
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        sm.h[le][q][a][k] = Hk[k];
        if constexpr (kLinear) {
          sm.p[le][q][a][k] = Hk[k];
          sm.q[le][q][a][k] = Hk[k];
        } else {
          sm.p[le][q][a][k] = Fi[0][k] * Hk[0] + Fi[1][k] * Hk[1] + Fi[2][k] * Hk[2];
          sm.q[le][q][a][k] = Fm[k][0] * Hk[0] + Fm[k][1] * Hk[1] + Fm[k][2] * Hk[2];
        }
      }
    }
  }
  if constexpr (kWantK) {
    sm.c[le][q][0] = tc.A;
    sm.c[le][q][1] = tc.hb;
    sm.c[le][q][2] = tc.c;
    sm.c[le][q][3] = tc.phi;
    __syncwarp();
    // ---- phase 2: blocks of the tile, summed over the 4 quadrature points
    const int n = (int)(task.w - task.z);
    for (int t = lane; t < n * 55; t += 32) {
      const int me = t / 55, slot = t - me * 55;
      const int a = c_pairs.a[slot], b = c_pairs.b[slot];
      KT acc[9];
#pragma unroll
      for (int j = 0; j < 9; ++j) acc[j] = (KT)0;
#pragma unroll
      for (int qq = 0; qq < 4; ++qq) {
        const KT cA = sm.c[me][qq][0], chb = sm.c[me][qq][1], cc = sm.c[me][qq][2], cphi = sm.c[me][qq][3];
        KT pa[3], pb[3], ha[3], ya[3], wb[3], s = 0;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          pa[k] = sm.p[me][qq][a][k];
          pb[k] = sm.p[me][qq][b][k];
          ha[k] = chb * pa[k];
          ya[k] = cc * sm.q[me][qq][a][k];
          wb[k] = cA * pb[k] + cc * sm.q[me][qq][b][k];
          s += sm.h[me][qq][a][k] * sm.h[me][qq][b][k];
        }
        s *= cphi;
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
          for (int m = 0; m < 3; ++m) acc[3 * k + m] += pa[k] * wb[m] + pb[k] * ha[m] + ya[k] * pb[m] + (k == m ? s : (KT)0);
      }
      const int64_t em = task.z + me;
      KT* rec = krec + (em & ring_mask) * L10::kK;
      if (slot < 45) {
        const int32_t ga = __ldg(A.conn + 10 * em + a), gb = __ldg(A.conn + 10 * em + b);
        store_pair_block<KT>(rec + L10::pair_off(slot), acc, ga > gb);
      } else {
        const KT dg[6] = {acc[0], acc[1], acc[2], acc[4], acc[5], acc[8]};
        store_diag_block<KT>(rec + L10::diag_off(slot - 45), dg);
      }
    }
  }
}

template <typename KT, int MODE>
__global__ void __launch_bounds__(kThreads10, 2)
tet10_persistent_kernel(Tet10Args A, GatherArgs g, QueueArgs Q, KT* __restrict__ krec, double* __restrict__ frec,
                        KT* __restrict__ k_out, double* __restrict__ f_out) {
  constexpr bool kWantF = (MODE & PSX_WANT_F) != 0;
  constexpr bool kWantK = (MODE & (PSX_WANT_K | PSX_LINEAR | PSX_MASS)) != 0;
  extern __shared__ __align__(16) unsigned char s_raw[];
  Tet10Smem<KT>& sm = reinterpret_cast<Tet10Smem<KT>*>(s_raw)[threadIdx.x >> 5];
  auto element_tile = [&](const int4& task) { tet10_tile<KT, MODE>(A, task, g.ring_mask, krec, frec, sm); };
  drain_queue<KT, 10, kWantK, kWantF, false, false>(g, Q, A.st, krec, frec, k_out, f_out, DRArgs{}, element_tile);
}

// det J and det F at the 4 quadrature points of one element (error messages).
__global__ void tet10_dets_kernel(const int32_t* __restrict__ conn, const double* __restrict__ X,
                                  const double* __restrict__ U, int64_t e, double* out8) {
  const int q = threadIdx.x;
  if (q >= 4) return;
  double L1, L2, L3;
  qp_coords(q, L1, L2, L3);
  double Jm[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, Fm[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int a = 0; a < 10; ++a) {
    double d[3];
    shape_grad(a, L1, L2, L3, d);
    const int64_t n = conn[10 * e + a];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) Jm[i][j] += X[3 * n + i] * d[j];
  }
  double Ji[3][3];
  const double detJ = inv3(Jm, Ji);
  if (U) {
    for (int a = 0; a < 10; ++a) {
      double d[3], H[3];
      shape_grad(a, L1, L2, L3, d);
      for (int j = 0; j < 3; ++j) H[j] = d[0] * Ji[0][j] + d[1] * Ji[1][j] + d[2] * Ji[2][j];
      const int64_t n = conn[10 * e + a];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Fm[i][j] += U[3 * n + i] * H[j];
    }
  }
  out8[2 * q] = detJ;
  out8[2 * q + 1] = det3(Fm);
}

template <typename KT, int MODE>
int run_tet10(const psx_plan_t* P, const Tet10Args& A, const WorkLayout& W, KT* k_out, double* f_out,
              cudaStream_t stream) {
  constexpr bool kWantK = (MODE & (PSX_WANT_K | PSX_LINEAR | PSX_MASS)) != 0;
  const GatherArgs g = gather_args(P, W.ring_elems);
  const QueueArgs Q = queue_args(P, W, kWantK);
  if (cudaMemsetAsync(W.counters, 0, W.counter_bytes, stream) != cudaSuccess) return PSX_ERR_CUDA;
  const size_t smem = sizeof(Tet10Smem<KT>) * (kThreads10 / 32);
  static unsigned long long s_smem_set = 0;
  if (set_dynamic_smem_once(tet10_persistent_kernel<KT, MODE>, (int)smem, &s_smem_set) != cudaSuccess)
    return PSX_ERR_CUDA;
  tet10_persistent_kernel<KT, MODE><<<W.grid, kThreads10, smem, stream>>>(A, g, Q, static_cast<KT*>(W.krec),
                                                                          W.frec, k_out, f_out);
  PSX_CUDA_CHECK_LAUNCH();
  return PSX_OK;
}

}  // namespace
}  // namespace psx

extern "C" int psx_tet10_assemble(const psx_plan_t* plan, const double* X, const double* u, const double* mu_e,
                                  const double* kappa_e, double mu, double kappa, double lam, int mode,
                                  int precision, double* f_out, void* k_out, void* work, int64_t work_bytes,
                                  void* status, void* stream) {
  using namespace psx;
  if (!plan || plan->npe != 10 || !X || !status || !work || plan->tile != kTile10) return PSX_ERR_ARG;
  const bool wantF = (mode & PSX_WANT_F) != 0, wantK = (mode & PSX_WANT_K) != 0,
             mass = (mode & PSX_MASS) != 0, linear = (mode & PSX_LINEAR) != 0 || mass;
  if (mode & ~(PSX_WANT_F | PSX_WANT_K | PSX_LINEAR | PSX_MASS)) return PSX_ERR_ARG;
  if ((mode & PSX_LINEAR) && mass) return PSX_ERR_ARG;
  if (linear && (wantF || wantK || !k_out)) return PSX_ERR_ARG;
  if (!linear && (!(wantF || wantK) || !u)) return PSX_ERR_ARG;
  if (wantF && !f_out) return PSX_ERR_ARG;
  if (wantK && !k_out) return PSX_ERR_ARG;
  WorkLayout W;
  int rc = work_layout(plan, precision, work, &W, 2, wantK || linear);
  if (rc != PSX_OK) return rc;
  if (work_bytes < W.total_bytes) return PSX_ERR_ARG;
  Tet10Args A{plan->conn, X, u, mu_e, kappa_e, mu, kappa, lam, static_cast<Status*>(status)};
  cudaStream_t s = static_cast<cudaStream_t>(stream);
#define PSX_T10(KT, M) run_tet10<KT, M>(plan, A, W, static_cast<KT*>(k_out), f_out, s)
  if (mass) return precision == PSX_FP64 ? PSX_T10(double, PSX_MASS) : PSX_T10(float, PSX_MASS);
  if (linear) return precision == PSX_FP64 ? PSX_T10(double, PSX_LINEAR) : PSX_T10(float, PSX_LINEAR);
  if (wantF && wantK)
    return precision == PSX_FP64 ? PSX_T10(double, PSX_WANT_F | PSX_WANT_K)
                                 : PSX_T10(float, PSX_WANT_F | PSX_WANT_K);
  if (wantK) return precision == PSX_FP64 ? PSX_T10(double, PSX_WANT_K) : PSX_T10(float, PSX_WANT_K);
  return PSX_T10(double, PSX_WANT_F);
#undef PSX_T10
}

extern "C" int psx_tet10_element_dets(const int32_t* conn, const double* X, const double* u, int64_t e,
                                      double* out8, void* stream) {
  if (!conn || !X || !out8 || e < 0) return PSX_ERR_ARG;
  psx::tet10_dets_kernel<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(conn, X, u, e, out8);
  PSX_CUDA_CHECK_LAUNCH();
  return PSX_OK;
}
