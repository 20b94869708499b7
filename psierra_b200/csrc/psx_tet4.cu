// Tet4 Total-Lagrangian NeoHookean assembly kernels for sm_100a.
//
// Replaces the per-element Python loops of SolidDomain (psierra domain/solid.py:172-207,
// 230-274, 280-325) around Tet4TotalLagrangian.compute_nonlinear_force_and_tangent_stiffness
// (element/tet4_total_lagrangian.py:77-139) and the COO->CSR / np.add.at scatter
// (utility/assembly.py:37-108).
//
// Owner-computes layout: one warp owns one node i and writes its three CSR rows and
// its three f entries exactly once.  Lane t of the warp evaluates incidence t of the
// node (element e holding i at local index a): the blocks K_ab (b = 0..3) and f_a.
// The blocks are staged in shared memory and lane r then sums, in ascending element
// order, every staged block whose neighbour rank is r.  Each output value is a
// fixed-order sum, so results are bitwise reproducible run to run; no atomics touch
// f or K.  Writes of a row are contiguous across lanes (lane r writes columns
// 3r..3r+2 of each of the three rows).
#include <cuda_runtime.h>
#include <stdint.h>

#include "psx_common.cuh"

namespace psx {
namespace {

constexpr int kWarps = 4;  // warps (nodes) per block

struct Tet4Geom {
  double g[4][3];  // shape-function gradients
  double V;        // reference volume
  double detD;     // det of [X1-X0 X2-X0 X3-X0] = det [1 X] of the reference
};

__device__ __forceinline__ void load_nodes(const double* __restrict__ A, int4 c, double out[4][3]) {
  const int ids[4] = {c.x, c.y, c.z, c.w};
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    const double* p = A + 3 * (int64_t)ids[b];
    out[b][0] = __ldg(p);
    out[b][1] = __ldg(p + 1);
    out[b][2] = __ldg(p + 2);
  }
}

// tet4_base.py:34-67 (A = [1 X], V = det A / 6, H = rows of A^-1) in the form
// D = [X1-X0 X2-X0 X3-X0], g_b = row b-1 of D^-1 (b >= 1), g_0 = -(g_1+g_2+g_3).
__device__ __forceinline__ void tet4_geometry(const double Xn[4][3], Tet4Geom& G) {
  double D[3][3], Di[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) D[i][j] = Xn[j + 1][i] - Xn[0][i];
  G.detD = inv3(D, Di);
  G.V = G.detD / 6.0;
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    G.g[1][j] = Di[0][j];
    G.g[2][j] = Di[1][j];
    G.g[3][j] = Di[2][j];
    G.g[0][j] = -(Di[0][j] + Di[1][j] + Di[2][j]);
  }
}

// Displacement gradient l = sum_b (u_b - u_0) g_b^T (exactly zero for a rigid translation).
__device__ __forceinline__ void tet4_grad(const double Un[4][3], const Tet4Geom& G, double l[3][3]) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      double v = 0.0;
#pragma unroll
      for (int b = 1; b < 4; ++b) v += (Un[b][i] - Un[0][i]) * G.g[b][j];
      l[i][j] = v;
    }
}

template <typename KT>
struct KStage {
  KT v[kWarps][32][37];  // 4 blocks x 9 values, padded
};

template <typename KT, int MODE>
__global__ void __launch_bounds__(kWarps * 32)
tet4_node_kernel(const int32_t* __restrict__ conn, const double* __restrict__ X, const double* __restrict__ U,
                 const double* __restrict__ mu_e, const double* __restrict__ kappa_e, double mu0,
                 double kappa0, double lam0, int32_t N, const int32_t* __restrict__ nbr_ptr,
                 const int32_t* __restrict__ inc_ptr, const int32_t* __restrict__ inc_elem,
                 const uint32_t* __restrict__ inc_code, double* __restrict__ f_out, KT* __restrict__ k_out,
                 Status* __restrict__ st) {
  constexpr bool kWantF = (MODE & PSX_WANT_F) != 0;
  constexpr bool kWantK = (MODE & (PSX_WANT_K | PSX_LINEAR)) != 0;
  constexpr bool kLinear = (MODE & PSX_LINEAR) != 0;
  __shared__ KStage<KT> sK;
  __shared__ double sF[kWarps][32][3];
  __shared__ uint32_t sCode[kWarps][32];

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int node = blockIdx.x * kWarps + warp;
  if (node >= N) return;  // uniform per warp
  const int i0 = inc_ptr[node], i1 = inc_ptr[node + 1];
  const int nb0 = nbr_ptr[node], deg = nbr_ptr[node + 1] - nb0;

  KT acc0[9], acc1[9];
  double facc[3];
#pragma unroll
  for (int j = 0; j < 9; ++j) acc0[j] = acc1[j] = (KT)0;
  facc[0] = facc[1] = facc[2] = 0.0;

  for (int c0 = i0; c0 < i1; c0 += 32) {
    const int cnt = min(32, i1 - c0);
    if (lane < cnt) {
      const int s = c0 + lane;
      const int e = inc_elem[s];
      const uint32_t code = inc_code[s];
      const int a = code & 3;
      const int4 cn = __ldg(reinterpret_cast<const int4*>(conn) + e);
      double Xn[4][3];
      load_nodes(X, cn, Xn);
      Tet4Geom G;
      tet4_geometry(Xn, G);
      const double mu = mu_e ? mu_e[e] : mu0;
      const double kappa = kappa_e ? kappa_e[e] : kappa0;
      if (a == 0 && !(G.detD > 0.0)) flag_bad_element(st, e, true);
      sCode[warp][lane] = code;

      // Own-node vectors are picked with selects so nothing is indexed at run time.
      double gad[3];
#pragma unroll
      for (int k = 0; k < 3; ++k)
        gad[k] = a == 0 ? G.g[0][k] : a == 1 ? G.g[1][k] : a == 2 ? G.g[2][k] : G.g[3][k];
      KT gk[4][3];
#pragma unroll
      for (int b = 0; b < 4; ++b)
#pragma unroll
        for (int k = 0; k < 3; ++k) gk[b][k] = (KT)G.g[b][k];
      const KT ga[3] = {(KT)gad[0], (KT)gad[1], (KT)gad[2]};

      if constexpr (kLinear) {
        // tet4_base.py:129-136: K_ab = V [lam g_a g_b^T + mu g_b g_a^T + mu (g_a.g_b) I]
        const KT Vl = (KT)(G.V * lam0), Vm = (KT)(G.V * mu0);
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          const KT s = Vm * (ga[0] * gk[b][0] + ga[1] * gk[b][1] + ga[2] * gk[b][2]);
#pragma unroll
          for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int m = 0; m < 3; ++m)
              sK.v[warp][lane][9 * b + 3 * k + m] =
                  Vl * ga[k] * gk[b][m] + Vm * gk[b][k] * ga[m] + (k == m ? s : (KT)0);
        }
      } else {
        double Un[4][3];
        load_nodes(U, cn, Un);
        double l[3][3];
        tet4_grad(Un, G, l);
        PointState ps;
        neohookean_point(l, mu, kappa, ps);
        if (a == 0 && G.detD > 0.0 && ps.Jm1 <= -1.0) flag_bad_element(st, e, false);
        if constexpr (kWantF) {
#pragma unroll
          for (int i = 0; i < 3; ++i)
            sF[warp][lane][i] = G.V * (ps.P[i][0] * gad[0] + ps.P[i][1] * gad[1] + ps.P[i][2] * gad[2]);
        }
        if constexpr (kWantK) {
          const TangentCoef<KT> tc = tangent_coef<KT>(ps, kappa, G.V);
          KT Fi[3][3], Fm[3][3];
#pragma unroll
          for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
              Fi[i][j] = (KT)ps.Finv[i][j];
              Fm[i][j] = (KT)ps.F[i][j];
            }
          // p_b = F^-T g_b, q_b = F g_b (KT arithmetic)
          KT p[4][3], q[4][3];
#pragma unroll
          for (int b = 0; b < 4; ++b)
#pragma unroll
            for (int k = 0; k < 3; ++k) {
              p[b][k] = Fi[0][k] * gk[b][0] + Fi[1][k] * gk[b][1] + Fi[2][k] * gk[b][2];
              q[b][k] = Fm[k][0] * gk[b][0] + Fm[k][1] * gk[b][1] + Fm[k][2] * gk[b][2];
            }
          KT pa[3], ha[3], ya[3];
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            pa[k] = a == 0 ? p[0][k] : a == 1 ? p[1][k] : a == 2 ? p[2][k] : p[3][k];
            const KT qa = a == 0 ? q[0][k] : a == 1 ? q[1][k] : a == 2 ? q[2][k] : q[3][k];
            ha[k] = tc.hb * pa[k];
            ya[k] = tc.c * qa;
          }
#pragma unroll
          for (int b = 0; b < 4; ++b) {
            KT wb[3];
#pragma unroll
            for (int m = 0; m < 3; ++m) wb[m] = tc.A * p[b][m] + tc.c * q[b][m];
            const KT s = tc.phi * (ga[0] * gk[b][0] + ga[1] * gk[b][1] + ga[2] * gk[b][2]);
#pragma unroll
            for (int k = 0; k < 3; ++k)
#pragma unroll
              for (int m = 0; m < 3; ++m)
                sK.v[warp][lane][9 * b + 3 * k + m] =
                    pa[k] * wb[m] + p[b][k] * ha[m] + ya[k] * p[b][m] + (k == m ? s : (KT)0);
          }
        }
      }
    }
    __syncwarp();
    // Fixed-order reduction: lane r owns neighbour columns r and r + 32.
    for (int t = 0; t < cnt; ++t) {
      const uint32_t code = sCode[warp][t];
      if constexpr (kWantK) {
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          const int rb = (code >> (2 + 7 * b)) & 127;
          if (rb == lane) {
#pragma unroll
            for (int j = 0; j < 9; ++j) acc0[j] += sK.v[warp][t][9 * b + j];
          } else if (rb == lane + 32) {
#pragma unroll
            for (int j = 0; j < 9; ++j) acc1[j] += sK.v[warp][t][9 * b + j];
          }
        }
      }
      if constexpr (kWantF && !kLinear) {
        if (lane == 0) {
          facc[0] += sF[warp][t][0];
          facc[1] += sF[warp][t][1];
          facc[2] += sF[warp][t][2];
        }
      }
    }
    __syncwarp();
  }

  if constexpr (kWantK) {
    const int64_t base = 9 * (int64_t)nb0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const int64_t row = base + 3 * (int64_t)deg * k;
      if (lane < deg) {
#pragma unroll
        for (int m = 0; m < 3; ++m) k_out[row + 3 * lane + m] = acc0[3 * k + m];
      }
      if (lane + 32 < deg) {
#pragma unroll
        for (int m = 0; m < 3; ++m) k_out[row + 3 * (lane + 32) + m] = acc1[3 * k + m];
      }
    }
  }
  if constexpr (kWantF && !kLinear) {
    if (lane == 0) {
      f_out[3 * (int64_t)node + 0] = facc[0];
      f_out[3 * (int64_t)node + 1] = facc[1];
      f_out[3 * (int64_t)node + 2] = facc[2];
    }
  }
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
int launch_tet4(const int32_t* conn, const double* X, const double* u, const double* mu_e,
                const double* kappa_e, double mu, double kappa, double lam, int64_t N, const int32_t* nbr_ptr,
                const int32_t* inc_ptr, const int32_t* inc_elem, const uint32_t* inc_code, double* f_out,
                void* k_out, void* status, cudaStream_t stream) {
  const unsigned blocks = (unsigned)((N + kWarps - 1) / kWarps);
  tet4_node_kernel<KT, MODE><<<blocks, kWarps * 32, 0, stream>>>(
      conn, X, u, mu_e, kappa_e, mu, kappa, lam, (int32_t)N, nbr_ptr, inc_ptr, inc_elem, inc_code, f_out,
      static_cast<KT*>(k_out), static_cast<Status*>(status));
  PSX_CUDA_CHECK_LAUNCH();
  return PSX_OK;
}

}  // namespace
}  // namespace psx

extern "C" size_t psx_status_bytes(void) { return sizeof(psx::Status); }

extern "C" int psx_tet4_assemble(const int32_t* conn, const double* X, const double* u, const double* mu_e,
                                 const double* kappa_e, double mu, double kappa, double lam, int64_t E,
                                 int64_t N, const int32_t* nbr_ptr, const int32_t* inc_ptr,
                                 const int32_t* inc_elem, const uint32_t* inc_code, int max_degree, int mode,
                                 int precision, double* f_out, void* k_out, void* status, void* stream) {
  using namespace psx;
  if (!conn || !X || !nbr_ptr || !inc_ptr || !inc_elem || !inc_code || !status) return PSX_ERR_ARG;
  if (E <= 0 || N <= 0 || N >= (int64_t)0x7fffffff || E >= (int64_t)0x7fffffff) return PSX_ERR_ARG;
  if (max_degree > PSX_TET4_MAX_DEGREE) return PSX_ERR_LIMIT;
  if (precision != PSX_FP64 && precision != PSX_FP32_MIXED) return PSX_ERR_ARG;
  const bool wantF = (mode & PSX_WANT_F) != 0, wantK = (mode & PSX_WANT_K) != 0,
             linear = (mode & PSX_LINEAR) != 0;
  if (linear && (wantF || wantK || !k_out)) return PSX_ERR_ARG;
  if (!linear && (!(wantF || wantK) || !u)) return PSX_ERR_ARG;
  if (wantF && !f_out) return PSX_ERR_ARG;
  if ((wantK || linear) && !k_out) return PSX_ERR_ARG;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
#define PSX_T4(KT, M) \
  launch_tet4<KT, M>(conn, X, u, mu_e, kappa_e, mu, kappa, lam, N, nbr_ptr, inc_ptr, inc_elem, inc_code, f_out, k_out, status, s)
  if (linear) return precision == PSX_FP64 ? PSX_T4(double, PSX_LINEAR) : PSX_T4(float, PSX_LINEAR);
  if (wantF && wantK)
    return precision == PSX_FP64 ? PSX_T4(double, PSX_WANT_F | PSX_WANT_K) : PSX_T4(float, PSX_WANT_F | PSX_WANT_K);
  if (wantK) return precision == PSX_FP64 ? PSX_T4(double, PSX_WANT_K) : PSX_T4(float, PSX_WANT_K);
  return PSX_T4(double, PSX_WANT_F);
#undef PSX_T4
}

extern "C" int psx_tet4_element_dets(const int32_t* conn, const double* X, const double* u, int64_t e,
                                     double* out2, void* stream) {
  if (!conn || !X || !out2 || e < 0) return PSX_ERR_ARG;
  psx::tet4_dets_kernel<<<1, 1, 0, static_cast<cudaStream_t>(stream)>>>(conn, X, u, e, out2);
  PSX_CUDA_CHECK_LAUNCH();
  return PSX_OK;
}
