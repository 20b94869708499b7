// Tet4 geometry and kinematics shared by the Tet4 kernels (assembly, K.v, adjoint,
// hyper-reduced evaluation).  element/tet4_base.py:34-67 and
// element/tet4_total_lagrangian.py:44-46 restated.
#pragma once

#include "psx_common.cuh"

namespace psx {

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
    for (int j = 0; j < 3; ++j) D[i][j] = dsub(Xn[j + 1][i], Xn[0][i]);
  G.detD = inv3(D, Di);
  G.V = G.detD / 6.0;
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    G.g[1][j] = Di[0][j];
    G.g[2][j] = Di[1][j];
    G.g[3][j] = Di[2][j];
    G.g[0][j] = -dadd(dadd(Di[0][j], Di[1][j]), Di[2][j]);
  }
}

// Displacement gradient l = sum_b (u_b - u_0) g_b^T (exactly zero for a rigid translation).
__device__ __forceinline__ void tet4_grad(const double Un[4][3], const Tet4Geom& G, double l[3][3]) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      l[i][j] = ddot3(dsub(Un[1][i], Un[0][i]), G.g[1][j], dsub(Un[2][i], Un[0][i]), G.g[2][j],
                      dsub(Un[3][i], Un[0][i]), G.g[3][j]);
    }
}

}  // namespace psx
