// Tet4 F-bar (nodal volume averaging) element and assembly for sm_100a.
//
// Restates psierra element/tet4_fbar.py: the nodal averages (:213-243)
//   v0_a = sum_{e in E_a} V_e / 4,   J_node_a = (sum_{e in E_a} V_e J_e / 4) / v0_a,
//   J_bar_e = mean of J_node over the element's nodes,
// the element force and deviatoric tangent at F_bar = (J_bar / J)^(1/3) F (:147-211,
// :375-410) and the nodal volumetric blocks kappa v0_a g_a g_a^T (:420-459).
//
// Closed forms (r = (J_bar/J)^(1/3); F, p_b = F^-T g_b, q_b = F g_b of the element's own
// deformation; S_bar, phi_bar = mu J_bar^(-2/3), I1_bar = tr(F_bar^T F_bar) at F_bar):
//   f_b = V F [r^2 S_bar + (1 - r^2) tr(S_bar)/3 I] g_b          (B_bar^T S_bar_voigt V)
//   K_bc = V [A' s_b s_c^T + B' (1/2 (p_b.p_c) I + 1/2 p_c p_b^T - 1/3 (t_b q_c^T + q_b t_c^T)
//             + 1/9 tr(C^-2) q_b q_c^T) + (g_b^T S_bar g_c) I]
// with s_b = p_b - tr(C^-1)/3 q_b, t_b = (F F^T)^-1 p_b, A' = kappa + 2/9 phi_bar I1_bar,
// B' = 2/3 phi_bar I1_bar - 2 kappa ln J_bar.  The reference's ratio^4 B_dev^T (C - kappa
// m m^T) B_dev contracts to this: B_dev maps to traceless strains, so kappa m m^T and the
// C^-1 (x) I terms of the NeoHookean tangent drop out, and the C^-1 scalings of C_bar
// cancel r^4.  The volumetric "div_e" rows (B_0 + B_1 + B_2) are q_b.
//
// Kernels (one thread per element, node, one-ring entry or two-ring block; every sum in
// the reference's order, ascending element / ascending patch node):
//   fbar_pre     V_e, J_e, q_e (and the inversion status)
//   fbar_nodes   v0_a, J_node_a
//   fbar_patch   g_a[b] = sum_{e in E_a, b in e} (V_e J_e / (4 v0_a)) q_e,b
//   fbar_element element record: 6 pair blocks, 4 diagonal blocks, 12 forces
//   fbar_gather  one-ring blocks and f (fixed-order sums of the records)
//   fbar_vol     two-ring blocks += sum_a kappa v0_a g_a[b] g_a[c]^T
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>

#include "psx_common.cuh"

namespace psx {
namespace {

constexpr int kFbThreads = 128;
constexpr int kFbRec = 6 * 9 + 4 * 6 + 12;  // doubles per element record

struct FbarArgs {
  const int32_t* conn;      // E x 4
  const double* X;
  const double* U;
  double mu, kappa;
  const int32_t* inc_ptr;   // N + 1: node -> incident elements, ascending
  const int32_t* inc_elem;
  const int32_t* nbr_ptr;   // one-ring graph (self included)
  const int32_t* nbr;
  const int32_t* blk_ptr;   // per one-ring entry: (e * 4 + a) * 4 + b, ascending e
  const int32_t* blk_src;
  const double* jbar_in;    // optional per-element J_bar (overrides the nodal average)
  double* V;                // E
  double* J;                // E
  double* q;                // 12 E
  double* v0;               // N
  double* Jn;               // N
  double* Jbar;             // E (output: the J_bar used)
  double* g;                // 3 x one-ring entries
  double* rec;              // kFbRec x E
  Status* st;
  int64_t E, N;
};

__device__ __forceinline__ void fb_nodes(const double* __restrict__ A, int4 c, double out[4][3]) {
  const int ids[4] = {c.x, c.y, c.z, c.w};
#pragma unroll
  for (int b = 0; b < 4; ++b)
#pragma unroll
    for (int k = 0; k < 3; ++k) out[b][k] = A[3 * (int64_t)ids[b] + k];
}

// D = [X1-X0, X2-X0, X3-X0]; g_b = rows of D^-1 (b >= 1), g_0 = -sum; V = det D / 6
__device__ __forceinline__ double fb_geometry(const double Xn[4][3], double g[4][3], double& detD) {
  double D[3][3], Di[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) D[i][j] = Xn[j + 1][i] - Xn[0][i];
  detD = inv3(D, Di);
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    g[1][j] = Di[0][j];
    g[2][j] = Di[1][j];
    g[3][j] = Di[2][j];
    g[0][j] = -(Di[0][j] + Di[1][j] + Di[2][j]);
  }
  return detD / 6.0;
}

__device__ __forceinline__ void fb_F(const double Un[4][3], const double g[4][3], double F[3][3]) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      double v = 0.0;
#pragma unroll
      for (int b = 1; b < 4; ++b) v += (Un[b][i] - Un[0][i]) * g[b][j];
      F[i][j] = (i == j ? 1.0 : 0.0) + v;
    }
}

__global__ void __launch_bounds__(kFbThreads) fbar_pre(FbarArgs A) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < A.E; e += (int64_t)gridDim.x * blockDim.x) {
    const int4 cn = reinterpret_cast<const int4*>(A.conn)[e];
    double Xn[4][3], Un[4][3], g[4][3], F[3][3], detD;
    fb_nodes(A.X, cn, Xn);
    fb_nodes(A.U, cn, Un);
    const double V = fb_geometry(Xn, g, detD);
    if (!(detD > 0.0)) flag_bad_element(A.st, e, true);
    fb_F(Un, g, F);
    const double J = det3(F);
    if (detD > 0.0 && !(J > 0.0)) flag_bad_element(A.st, e, false);
    A.V[e] = V;
    A.J[e] = J;
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
      for (int k = 0; k < 3; ++k) A.q[12 * e + 3 * b + k] = F[k][0] * g[b][0] + F[k][1] * g[b][1] + F[k][2] * g[b][2];
  }
}

// np.bincount of 0.25 V_e and 0.25 V_e J_e over the element-major node list (ascending e)
__global__ void __launch_bounds__(kFbThreads) fbar_nodes(FbarArgs A) {
  for (int64_t a = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; a < A.N; a += (int64_t)gridDim.x * blockDim.x) {
    double v0 = 0.0, v = 0.0;
    for (int32_t s = A.inc_ptr[a]; s < A.inc_ptr[a + 1]; ++s) {
      const int32_t e = A.inc_elem[s];
      const double w = 0.25 * A.V[e];
      v0 += w;
      v += w * A.J[e];
    }
    A.v0[a] = v0;
    A.Jn[a] = v / v0;  // isolated nodes never enter an element average
  }
}

// g_a[b] for every one-ring entry (a, b): thread per node a
// One thread per one-ring entry t (node a and its neighbour; a found by a binary search
// of nbr_ptr), so that a warp writes consecutive entries.
__global__ void __launch_bounds__(kFbThreads) fbar_patch(FbarArgs A) {
  const int64_t n1 = A.nbr_ptr[A.N];
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n1; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t lo = 0, hi = A.N;  // nbr_ptr[lo] <= t < nbr_ptr[hi]
    while (hi - lo > 1) {
      const int64_t mid = (lo + hi) / 2;
      if (A.nbr_ptr[mid] <= t)
        lo = mid;
      else
        hi = mid;
    }
    const double v0 = A.v0[lo];
    double g0 = 0.0, g1 = 0.0, g2 = 0.0;
    for (int32_t s = A.blk_ptr[t]; s < A.blk_ptr[t + 1]; ++s) {
      const int32_t code = A.blk_src[s];
      const int32_t lb = code & 3;
      const int64_t e = code >> 4;
      const double w = 0.25 * A.V[e] * A.J[e] / v0;
      const double* qe = A.q + 12 * e + 3 * lb;
      g0 += w * qe[0];
      g1 += w * qe[1];
      g2 += w * qe[2];
    }
    A.g[3 * t] = g0;
    A.g[3 * t + 1] = g1;
    A.g[3 * t + 2] = g2;
  }
}

__global__ void __launch_bounds__(kFbThreads) fbar_element(FbarArgs A) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < A.E; e += (int64_t)gridDim.x * blockDim.x) {
    const int4 cn = reinterpret_cast<const int4*>(A.conn)[e];
    double Xn[4][3], Un[4][3], g[4][3], F[3][3], detD;
    fb_nodes(A.X, cn, Xn);
    fb_nodes(A.U, cn, Un);
    const double V = fb_geometry(Xn, g, detD);
    fb_F(Un, g, F);
    const double J = det3(F);
    const double jbar = A.jbar_in ? A.jbar_in[e] : (A.Jn[cn.x] + A.Jn[cn.y] + A.Jn[cn.z] + A.Jn[cn.w]) / 4.0;
    A.Jbar[e] = jbar;
    const double r = pow(jbar / J, 1.0 / 3.0);
    // NeoHookean at F_bar = r F (neohookean.py:74-92): S_bar = C_bar^-1 (2 phi dev E_bar + beta I)
    double Fb[3][3], Fbi[3][3], Fi[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) Fb[i][j] = r * F[i][j];
    const double Jb = inv3(Fb, Fbi);
    inv3(F, Fi);
    double Eb[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const double c = Fb[0][i] * Fb[0][j] + Fb[1][i] * Fb[1][j] + Fb[2][i] * Fb[2][j];
        Eb[i][j] = 0.5 * (c - (i == j ? 1.0 : 0.0));
      }
    const double I1b = 3.0 + 2.0 * (Eb[0][0] + Eb[1][1] + Eb[2][2]);
    const double lnJb = log(Jb);
    const double phib = A.mu * exp((-2.0 / 3.0) * lnJb);
    const double betab = A.kappa * lnJb;
    const double trEb = Eb[0][0] + Eb[1][1] + Eb[2][2];
    double T[3][3], Cbi[3][3], Sb[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        T[i][j] = 2.0 * phib * (Eb[i][j] - (i == j ? trEb / 3.0 : 0.0)) + (i == j ? betab : 0.0);
        Cbi[i][j] = Fbi[i][0] * Fbi[j][0] + Fbi[i][1] * Fbi[j][1] + Fbi[i][2] * Fbi[j][2];
      }
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) Sb[i][j] = Cbi[i][0] * T[0][j] + Cbi[i][1] * T[1][j] + Cbi[i][2] * T[2][j];
    // symmetrise (S_bar is symmetric; the product above is exact up to rounding)
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = i + 1; j < 3; ++j) {
        const double m = 0.5 * (Sb[i][j] + Sb[j][i]);
        Sb[i][j] = m;
        Sb[j][i] = m;
      }
    const double trS = Sb[0][0] + Sb[1][1] + Sb[2][2];
    // per node: p = F^-T g, q = F g, t = (F F^T)^-1 p = F^-T F^-1 p, s = p - tr(C^-1)/3 q
    double p[4][3], qv[4][3], t[4][3], s[4][3];
    double Ci[3][3];  // C^-1 = F^-1 F^-T
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) Ci[i][j] = Fi[i][0] * Fi[j][0] + Fi[i][1] * Fi[j][1] + Fi[i][2] * Fi[j][2];
    const double trCi = Ci[0][0] + Ci[1][1] + Ci[2][2];
    double trCi2 = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) trCi2 += Ci[i][j] * Ci[j][i];
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      double fp[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        p[b][k] = Fi[0][k] * g[b][0] + Fi[1][k] * g[b][1] + Fi[2][k] * g[b][2];
        qv[b][k] = F[k][0] * g[b][0] + F[k][1] * g[b][1] + F[k][2] * g[b][2];
      }
#pragma unroll
      for (int k = 0; k < 3; ++k) fp[k] = Fi[k][0] * p[b][0] + Fi[k][1] * p[b][1] + Fi[k][2] * p[b][2];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        t[b][k] = Fi[0][k] * fp[0] + Fi[1][k] * fp[1] + Fi[2][k] * fp[2];
        s[b][k] = p[b][k] - (trCi / 3.0) * qv[b][k];
      }
    }
    const double Ap = A.kappa + (2.0 / 9.0) * phib * I1b;
    const double Bp = (2.0 / 3.0) * phib * I1b - 2.0 * A.kappa * lnJb;
    double* R = A.rec + (int64_t)kFbRec * e;
    const int gid[4] = {cn.x, cn.y, cn.z, cn.w};
    int slot = 0;
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = a; b < 4; ++b) {
        double gsg = 0.0, pp = 0.0;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          pp += p[a][i] * p[b][i];
#pragma unroll
          for (int j = 0; j < 3; ++j) gsg += g[a][i] * Sb[i][j] * g[b][j];
        }
        double v[3][3];
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
          for (int m = 0; m < 3; ++m) {
            double x = Ap * s[a][k] * s[b][m] +
                       Bp * (0.5 * p[b][k] * p[a][m] - (t[a][k] * qv[b][m] + qv[a][k] * t[b][m]) / 3.0 +
                             (trCi2 / 9.0) * qv[a][k] * qv[b][m]);
            if (k == m) x += Bp * 0.5 * pp + gsg;
            v[k][m] = V * x;
          }
        if (a == b) {
          double* d = R + 54 + 6 * a;
          d[0] = v[0][0]; d[1] = v[0][1]; d[2] = v[0][2]; d[3] = v[1][1]; d[4] = v[1][2]; d[5] = v[2][2];
        } else {
          double* o = R + 9 * slot;
          const bool swap = gid[a] > gid[b];  // rows = the node of smaller global id
#pragma unroll
          for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int m = 0; m < 3; ++m) o[3 * k + m] = swap ? v[m][k] : v[k][m];
          ++slot;
        }
      }
    // f_b = V F [r^2 S_bar + (1 - r^2) tr(S_bar)/3 I] g_b
    const double r2 = r * r;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      double w[3];
#pragma unroll
      for (int i = 0; i < 3; ++i)
        w[i] = r2 * (Sb[i][0] * g[b][0] + Sb[i][1] * g[b][1] + Sb[i][2] * g[b][2]) +
               (1.0 - r2) * (trS / 3.0) * g[b][i];
#pragma unroll
      for (int k = 0; k < 3; ++k) R[78 + 3 * b + k] = V * (F[k][0] * w[0] + F[k][1] * w[1] + F[k][2] * w[2]);
    }
  }
}

struct FbarGather {
  const int32_t* pair_info2;  // 4 per one-ring pair: positions in the two-ring CSR
  const int32_t* pair_ptr;
  const int32_t* pair_src;    // e * 64 + local pair slot
  const int32_t* node_info2;
  const int32_t* node_ptr;
  const int32_t* node_src;    // e * 16 + local node
  int64_t n_pairs, n_nodes;
};

__global__ void __launch_bounds__(kFbThreads) fbar_gather(FbarGather G, const double* __restrict__ rec,
                                                          double* __restrict__ k_out, double* __restrict__ f_out) {
  const int64_t total = G.n_pairs + G.n_nodes;
  for (int64_t it = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; it < total; it += (int64_t)gridDim.x * blockDim.x) {
    if (it < G.n_pairs) {
      if (!k_out) continue;
      const int32_t* info = G.pair_info2 + 4 * it;
      double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      for (int32_t s = G.pair_ptr[it]; s < G.pair_ptr[it + 1]; ++s) {
        const int32_t c = G.pair_src[s];
        const double* o = rec + (int64_t)kFbRec * (c >> 6) + 9 * (c & 63);
#pragma unroll
        for (int j = 0; j < 9; ++j) acc[j] += o[j];
      }
#pragma unroll
      for (int k = 0; k < 3; ++k) store3(k_out + info[0] + (int64_t)info[1] * k, acc[3 * k], acc[3 * k + 1], acc[3 * k + 2]);
#pragma unroll
      for (int m = 0; m < 3; ++m) store3(k_out + info[2] + (int64_t)info[3] * m, acc[m], acc[3 + m], acc[6 + m]);
    } else {
      const int64_t n = it - G.n_pairs;
      const int32_t* info = G.node_info2 + 4 * n;
      double d[6] = {0, 0, 0, 0, 0, 0}, f[3] = {0, 0, 0};
      for (int32_t s = G.node_ptr[n]; s < G.node_ptr[n + 1]; ++s) {
        const int32_t c = G.node_src[s];
        const double* R = rec + (int64_t)kFbRec * (c >> 4);
        const int a = c & 15;
#pragma unroll
        for (int j = 0; j < 6; ++j) d[j] += R[54 + 6 * a + j];
#pragma unroll
        for (int k = 0; k < 3; ++k) f[k] += R[78 + 3 * a + k];
      }
      if (k_out && info[1] > 0) {
        const double full[9] = {d[0], d[1], d[2], d[1], d[3], d[4], d[2], d[4], d[5]};
#pragma unroll
        for (int k = 0; k < 3; ++k)
          store3(k_out + info[0] + (int64_t)info[1] * k, full[3 * k], full[3 * k + 1], full[3 * k + 2]);
      }
      if (f_out) store3(f_out + 3 * (int64_t)info[2], f[0], f[1], f[2]);
    }
  }
}

// two-ring block (b, c): K += sum_a (kappa v0_a) (g_a[b] g_a[c]^T), a ascending.  One
// thread per two-ring entry t (the block of node b and its t-th two-ring neighbour; b
// found by a binary search of nbr2_ptr), so that the threads of a warp update adjacent
// blocks of the same rows.
__global__ void __launch_bounds__(kFbThreads) fbar_vol(int64_t N, const int32_t* __restrict__ nbr2_ptr,
                                                       const int32_t* __restrict__ vol_ptr,
                                                       const int32_t* __restrict__ vol_src,
                                                       const double* __restrict__ v0, const double* __restrict__ g,
                                                       double kappa, double* __restrict__ k_out) {
  const int64_t n2 = nbr2_ptr[N];
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n2; t += (int64_t)gridDim.x * blockDim.x) {
    // the node b with nbr2_ptr[b] <= t < nbr2_ptr[b + 1]
    int64_t lo = 0, hi = N;
    while (hi - lo > 1) {
      const int64_t mid = (lo + hi) / 2;
      if (nbr2_ptr[mid] <= t)
        lo = mid;
      else
        hi = mid;
    }
    const int64_t b = lo;
    const int32_t t0 = nbr2_ptr[b], t1 = nbr2_ptr[b + 1];
    const int64_t row = 9 * (int64_t)t0, stride = 3 * (int64_t)(t1 - t0);
    double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int32_t s = vol_ptr[t]; s < vol_ptr[t + 1]; ++s) {
      const int32_t* v = vol_src + 3 * (int64_t)s;
      const double sc = kappa * v0[v[0]];
      const double* gb = g + 3 * (int64_t)v[1];
      const double* gc = g + 3 * (int64_t)v[2];
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int m = 0; m < 3; ++m) acc[3 * k + m] += sc * (gb[k] * gc[m]);
    }
    const int64_t col = 3 * (t - t0);
#pragma unroll
    for (int k = 0; k < 3; ++k) add3(k_out + row + stride * k + col, acc[3 * k], acc[3 * k + 1], acc[3 * k + 2]);
  }
}

// Single elements with given J_bar (Tet4Fbar.compute_nonlinear_force_and_tangent_stiffness,
// element/tet4_fbar.py:147-211): k = B_bar^T C B_bar V + G^T (I (x) S_bar) G V with the full
// Voigt tangent C of NeoHookean at F_bar (material/neohookean.py:95-120, Voigt order
// xx yy zz xy yz zx), B the nonlinear strain-displacement matrix and
// B_bar = r^2 (B - m b_vol^T) + m b_vol^T.  An API-compatibility path: one thread per
// element, explicit 6 x 12 products.
__global__ void __launch_bounds__(kFbThreads) fbar_single(int64_t n, const double* __restrict__ Xe,
                                                          const double* __restrict__ Ue,
                                                          const double* __restrict__ jbar, double mu, double kappa,
                                                          double* __restrict__ k_out, double* __restrict__ f_out,
                                                          Status* st) {
  constexpr int vi[6] = {0, 1, 2, 0, 1, 2}, vj[6] = {0, 1, 2, 1, 2, 0};
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    double Xn[4][3], Un[4][3], g[4][3], F[3][3], detD;
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        Xn[b][k] = Xe[12 * e + 3 * b + k];
        Un[b][k] = Ue[12 * e + 3 * b + k];
      }
    const double V = fb_geometry(Xn, g, detD);
    if (!(detD > 0.0)) flag_bad_element(st, e, true);
    fb_F(Un, g, F);
    const double J = det3(F);
    if (detD > 0.0 && !(J > 0.0)) flag_bad_element(st, e, false);
    const double r = pow(jbar[e] / J, 1.0 / 3.0);
    double Fb[3][3], C[3][3], Ci[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) Fb[i][j] = r * F[i][j];
    const double Jb = det3(Fb);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) C[i][j] = Fb[0][i] * Fb[0][j] + Fb[1][i] * Fb[1][j] + Fb[2][i] * Fb[2][j];
    inv3(C, Ci);
    const double I1 = C[0][0] + C[1][1] + C[2][2];
    const double fac = mu * pow(Jb, -2.0 / 3.0);
    const double lnJ = log(Jb);
    double S[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) S[i][j] = fac * ((i == j ? 1.0 : 0.0) - I1 / 3.0 * Ci[i][j]) + kappa * lnJ * Ci[i][j];
    double Cv[6][6];
    for (int a = 0; a < 6; ++a)
      for (int b = 0; b < 6; ++b) {
        const int i = vi[a], j = vj[a], k = vi[b], l = vj[b];
        const double oo = Ci[i][j] * Ci[k][l];
        const double ii = 0.5 * (Ci[i][k] * Ci[j][l] + Ci[i][l] * Ci[j][k]);
        const double ci = Ci[i][j] * (k == l ? 1.0 : 0.0) + (i == j ? 1.0 : 0.0) * Ci[k][l];
        Cv[a][b] = kappa * oo - 2.0 * kappa * lnJ * ii - (2.0 / 3.0) * fac * ci + (2.0 / 9.0) * fac * I1 * oo +
                   (2.0 / 3.0) * fac * I1 * ii;
      }
    double Bb[6][12];
    for (int b = 0; b < 4; ++b)
      for (int k = 0; k < 3; ++k) {
        double col[6];
        for (int a = 0; a < 6; ++a) {
          const int i = vi[a], j = vj[a];
          col[a] = i == j ? F[k][i] * g[b][i] : F[k][i] * g[b][j] + F[k][j] * g[b][i];
        }
        const double bvol = (col[0] + col[1] + col[2]) / 3.0;
        for (int a = 0; a < 6; ++a) {
          const double m = a < 3 ? 1.0 : 0.0;
          Bb[a][3 * b + k] = r * r * (col[a] - m * bvol) + m * bvol;
        }
      }
    double CB[6][12];
    for (int a = 0; a < 6; ++a)
      for (int c = 0; c < 12; ++c) {
        double x = 0.0;
        for (int b = 0; b < 6; ++b) x += Cv[a][b] * Bb[b][c];
        CB[a][c] = x;
      }
    const double Sv[6] = {S[0][0], S[1][1], S[2][2], S[0][1], S[1][2], S[2][0]};
    for (int c = 0; c < 12; ++c) {
      double fv = 0.0;
      for (int a = 0; a < 6; ++a) fv += Bb[a][c] * Sv[a];
      f_out[12 * e + c] = fv * V;
      for (int d = 0; d < 12; ++d) {
        double x = 0.0;
        for (int a = 0; a < 6; ++a) x += Bb[a][c] * CB[a][d];
        double geo = 0.0;
        if (c % 3 == d % 3) {
          const int pa = c / 3, pb = d / 3;
          for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) geo += g[pa][i] * S[i][j] * g[pb][j];
        }
        k_out[144 * e + 12 * c + d] = x * V + geo * V;
      }
    }
  }
}

inline int fb_grid(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + kFbThreads - 1) / kFbThreads, 148 * 16)); }

}  // namespace
}  // namespace psx

extern "C" int psx_fbar_element(int64_t n, const double* X_elem, const double* u_elem, const double* jbar, double mu,
                                double kappa, double* k_out, double* f_out, void* status, void* stream) {
  using namespace psx;
  if (n <= 0 || !X_elem || !u_elem || !jbar || !k_out || !f_out || !status) return PSX_ERR_ARG;
  fbar_single<<<fb_grid(n), kFbThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      n, X_elem, u_elem, jbar, mu, kappa, k_out, f_out, static_cast<Status*>(status));
  PSX_CUDA_CHECK_LAUNCH();
  return PSX_OK;
}

extern "C" int64_t psx_fbar_work_doubles(int64_t E, int64_t N, int64_t n_nbr) {
  return 3 * E + 12 * E + 2 * N + E + 3 * n_nbr + (int64_t)psx::kFbRec * E;
}

extern "C" int psx_fbar_assemble(const int32_t* conn, int64_t E, int64_t N, const double* X, const double* u,
                                 double mu, double kappa, const int32_t* inc_ptr, const int32_t* inc_elem,
                                 const int32_t* nbr_ptr, const int32_t* nbr, int64_t n_nbr, const int32_t* blk_ptr,
                                 const int32_t* blk_src, int64_t n_pairs, const int32_t* pair_info2,
                                 const int32_t* pair_ptr, const int32_t* pair_src, const int32_t* node_info2,
                                 const int32_t* node_ptr, const int32_t* node_src, const int32_t* nbr2_ptr,
                                 const int32_t* vol_ptr, const int32_t* vol_src, const double* jbar_in,
                                 double* f_out, double* k_out, int64_t nnz2, double* jbar_out, double* work,
                                 int64_t work_doubles, void* status, void* stream) {
  using namespace psx;
  if (!conn || E <= 0 || N <= 0 || !X || !u || !inc_ptr || !inc_elem || !nbr_ptr || !nbr || !blk_ptr || !blk_src ||
      !pair_info2 || !pair_ptr || !pair_src || !node_info2 || !node_ptr || !node_src || !nbr2_ptr || !vol_ptr ||
      !vol_src || !work || !status || (!f_out && !k_out))
    return PSX_ERR_ARG;
  if (work_doubles < psx_fbar_work_doubles(E, N, n_nbr) || (k_out && nnz2 <= 0)) return PSX_ERR_ARG;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  FbarArgs A;
  A.conn = conn; A.X = X; A.U = u; A.mu = mu; A.kappa = kappa;
  A.inc_ptr = inc_ptr; A.inc_elem = inc_elem; A.nbr_ptr = nbr_ptr; A.nbr = nbr;
  A.blk_ptr = blk_ptr; A.blk_src = blk_src; A.jbar_in = jbar_in;
  double* w = work;
  A.V = w; w += E;
  A.J = w; w += E;
  A.Jbar = jbar_out ? jbar_out : w; w += E;
  A.q = w; w += 12 * E;
  A.v0 = w; w += N;
  A.Jn = w; w += N;
  A.g = w; w += 3 * n_nbr;
  A.rec = w;
  A.st = static_cast<Status*>(status);
  A.E = E; A.N = N;
  fbar_pre<<<fb_grid(E), kFbThreads, 0, s>>>(A);
  fbar_nodes<<<fb_grid(N), kFbThreads, 0, s>>>(A);
  if (k_out) fbar_patch<<<fb_grid(n_nbr), kFbThreads, 0, s>>>(A);  // one thread per one-ring entry
  fbar_element<<<fb_grid(E), kFbThreads, 0, s>>>(A);
  if (k_out && cudaMemsetAsync(k_out, 0, sizeof(double) * nnz2, s) != cudaSuccess) return PSX_ERR_CUDA;
  FbarGather G{pair_info2, pair_ptr, pair_src, node_info2, node_ptr, node_src, n_pairs, N};
  fbar_gather<<<fb_grid(n_pairs + N), kFbThreads, 0, s>>>(G, A.rec, k_out, f_out);
  // one thread per two-ring entry: the two-ring CSR holds 9 values per entry
  if (k_out) fbar_vol<<<fb_grid(nnz2 / 9), kFbThreads, 0, s>>>(N, nbr2_ptr, vol_ptr, vol_src, A.v0, A.g, kappa, k_out);
  PSX_CUDA_CHECK_LAUNCH();
  return PSX_OK;
}
