// Hyper-reduced (ECSW) Tet4 evaluation for sm_100a.
//
// Restates HyperReducedECSWModel.evaluate_forces_and_stiffness (psierra
// hyperreduction/model.py:254-318): on the reduced integration domain (p elements with
// cubature weights w_e and modal sub-bases Phi_e, 12 x r),
//   u_e = Phi_e u_r,  f_r = sum_e w_e Phi_e^T f_e(u_e),  K_r = sum_e w_e Phi_e^T k_e(u_e) Phi_e,
//   K_r <- (K_r + K_r^T) / 2.
// ecsw_elements: one thread per element -- u_e, the element's dense k and f from the
// closed-form NeoHookean Tet4 tangent of the assembly kernels, T_e = w_e k_e Phi_e and
// v_e = w_e f_e.  ecsw_reduce: one thread per (i, j) of the r x r result, summing over the
// elements in ascending order (fixed order, reproducible), and the symmetrisation.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "psx_common.cuh"
#include "psx_tet4_math.cuh"

namespace psx {
namespace {

constexpr int kEcThreads = 128;

__global__ void __launch_bounds__(kEcThreads) ecsw_elements(int64_t n, int32_t r, const double* __restrict__ Xe,
                                                            const double* __restrict__ phi,
                                                            const double* __restrict__ w,
                                                            const double* __restrict__ ur,
                                                            const double* __restrict__ mu_e,
                                                            const double* __restrict__ kappa_e, double mu0,
                                                            double kappa0, double* __restrict__ T,
                                                            double* __restrict__ v, Status* st) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const double* P = phi + (int64_t)12 * r * e;  // row-major 12 x r
    double Xn[4][3], Un[4][3];
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        Xn[b][k] = Xe[12 * e + 3 * b + k];
        double s = 0.0;
        for (int j = 0; j < r; ++j) s += P[(3 * b + k) * r + j] * ur[j];
        Un[b][k] = s;
      }
    Tet4Geom G;
    tet4_geometry(Xn, G);
    if (!(G.detD > 0.0)) flag_bad_element(st, e, true);
    double l[3][3];
    tet4_grad(Un, G, l);
    PointState ps;
    const double mu = mu_e ? mu_e[e] : mu0, kappa = kappa_e ? kappa_e[e] : kappa0;
    neohookean_point(l, mu, kappa, ps);
    if (G.detD > 0.0 && ps.Jm1 <= -1.0) flag_bad_element(st, e, false);
    const double we = w[e];
    // f_a = V P g_a
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int i = 0; i < 3; ++i)
        v[12 * e + 3 * a + i] =
            we * (G.V * (ps.P[i][0] * G.g[a][0] + ps.P[i][1] * G.g[a][1] + ps.P[i][2] * G.g[a][2]));
    const TangentCoef<double> tc = tangent_coef<double>(ps, kappa, G.V);
    double p[4][3], q[4][3];
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        p[b][k] = ps.Finv[0][k] * G.g[b][0] + ps.Finv[1][k] * G.g[b][1] + ps.Finv[2][k] * G.g[b][2];
        q[b][k] = ps.F[k][0] * G.g[b][0] + ps.F[k][1] * G.g[b][1] + ps.F[k][2] * G.g[b][2];
      }
    // T = w k Phi, row (a, k) of k: K_ab[k][m] over (b, m)
    for (int a = 0; a < 4; ++a)
      for (int k = 0; k < 3; ++k) {
        double krow[12];
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          const double gg = G.g[a][0] * G.g[b][0] + G.g[a][1] * G.g[b][1] + G.g[a][2] * G.g[b][2];
#pragma unroll
          for (int m = 0; m < 3; ++m)
            krow[3 * b + m] = tc.A * p[a][k] * p[b][m] + tc.hb * p[b][k] * p[a][m] +
                              tc.c * (p[a][k] * q[b][m] + q[a][k] * p[b][m]) + (k == m ? tc.phi * gg : 0.0);
        }
        double* Trow = T + (int64_t)12 * r * e + (3 * a + k) * (int64_t)r;
        for (int j = 0; j < r; ++j) {
          double s = 0.0;
#pragma unroll
          for (int d = 0; d < 12; ++d) s += krow[d] * P[d * r + j];
          Trow[j] = we * s;
        }
      }
  }
}

__global__ void __launch_bounds__(kEcThreads) ecsw_reduce(int64_t n, int32_t r, const double* __restrict__ phi,
                                                          const double* __restrict__ T,
                                                          const double* __restrict__ v, double* __restrict__ f_r,
                                                          double* __restrict__ K_r) {
  const int64_t total = (int64_t)r * r + r;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    if (t >= (int64_t)r * r) {
      const int i = (int)(t - (int64_t)r * r);
      double s = 0.0;
      for (int64_t e = 0; e < n; ++e) {
        const double* P = phi + (int64_t)12 * r * e;
        for (int a = 0; a < 12; ++a) s += P[a * r + i] * v[12 * e + a];
      }
      f_r[i] = s;
      continue;
    }
    const int i = (int)(t / r), j = (int)(t % r);
    double sij = 0.0, sji = 0.0;
    for (int64_t e = 0; e < n; ++e) {
      const double* P = phi + (int64_t)12 * r * e;
      const double* Te = T + (int64_t)12 * r * e;
      for (int a = 0; a < 12; ++a) {
        sij += P[a * r + i] * Te[a * r + j];
        sji += P[a * r + j] * Te[a * r + i];
      }
    }
    K_r[(int64_t)i * r + j] = 0.5 * (sij + sji);
  }
}

inline int ec_grid(int64_t n) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((n + kEcThreads - 1) / kEcThreads, 148 * 8));
}

}  // namespace
}  // namespace psx

extern "C" int64_t psx_ecsw_work_doubles(int64_t n, int32_t r) { return (int64_t)12 * r * n + 12 * n; }

extern "C" int psx_ecsw_evaluate(int64_t n, int32_t r, const double* X_elem, const double* phi_elem,
                                 const double* weights, const double* u_r, const double* mu_e, const double* kappa_e,
                                 double mu, double kappa, double* f_r, double* K_r, double* work,
                                 int64_t work_doubles, void* status, void* stream) {
  using namespace psx;
  if (n <= 0 || r <= 0 || !X_elem || !phi_elem || !weights || !u_r || !f_r || !K_r || !work || !status)
    return PSX_ERR_ARG;
  if ((mu_e == nullptr) != (kappa_e == nullptr)) return PSX_ERR_ARG;
  if (work_doubles < psx_ecsw_work_doubles(n, r)) return PSX_ERR_ARG;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double* T = work;
  double* v = work + (int64_t)12 * r * n;
  ecsw_elements<<<ec_grid(n), kEcThreads, 0, s>>>(n, r, X_elem, phi_elem, weights, u_r, mu_e, kappa_e, mu, kappa, T,
                                                 v, static_cast<Status*>(status));
  ecsw_reduce<<<ec_grid((int64_t)r * r + r), kEcThreads, 0, s>>>(n, r, phi_elem, T, v, f_r, K_r);
  PSX_CUDA_CHECK_LAUNCH();
  return PSX_OK;
}
