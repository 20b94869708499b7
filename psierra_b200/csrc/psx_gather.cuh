// Owner-computes gather of element records into the CSR values and f (kernel "B").
//
// The element kernel writes, per element e, a record into a ring of scratch slots
// (slot = e & ring_mask):
//   K part (KT): npair off-diagonal 3x3 blocks, 12 values each (9 used), oriented with
//                rows = the element node of smaller global id; then npe diagonal blocks,
//                8 values each (xx xy xz yy yz zz + 2 pad).  npair = npe (npe - 1) / 2.
//   f part (double): 3 values per element node.
// A pair item (i < j) sums the blocks of every element holding both nodes, in
// ascending element order, and writes K_ij (row 3i+k, upper) and its transpose K_ji
// (row 3j+m, lower).  A node item sums the diagonal blocks and f contributions of its
// incident elements.  Each output value is written once, as a fixed-order sum: the
// reference's COO->CSR duplicate summation (psierra utility/assembly.py:75-76) and
// np.add.at (utility/assembly.py:103-107), without atomics.
#pragma once

#include "psx_common.cuh"

namespace psx {

template <int NPE>
struct RecLayout {
  static constexpr int kPairs = NPE * (NPE - 1) / 2;
  static constexpr int kK = kPairs * 12 + NPE * 8;  // KT values per element record
  static constexpr int kF = NPE * 3;                 // doubles per element f record
  __host__ __device__ static constexpr int pair_off(int slot) { return slot * 12; }
  __host__ __device__ static constexpr int diag_off(int a) { return kPairs * 12 + a * 8; }
};

struct GatherArgs {
  const int32_t* pair_info;  // 4 per pair: pos_up, stride_up, pos_lo, stride_lo
  const int32_t* pair_ptr;
  const int32_t* pair_src;   // e * 64 + local pair slot
  const int32_t* node_info;  // 4 per node item: pos_d, stride, node, pad
  const int32_t* node_ptr;
  const int32_t* node_src;   // e * 16 + local node index
  int32_t p0, p1;            // pair item range of this launch
  int32_t n0, n1;            // node item range of this launch
  int64_t ring_mask;
};

template <typename KT>
__device__ __forceinline__ void load12(const KT* __restrict__ p, KT v[12]) {
  if constexpr (sizeof(KT) == 4) {
    const float4* q = reinterpret_cast<const float4*>(p);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      float4 t = __ldcg(q + i);
      v[4 * i] = t.x; v[4 * i + 1] = t.y; v[4 * i + 2] = t.z; v[4 * i + 3] = t.w;
    }
  } else {
    const double2* q = reinterpret_cast<const double2*>(p);
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      double2 t = __ldcg(q + i);
      v[2 * i] = t.x; v[2 * i + 1] = t.y;
    }
  }
}

template <typename KT>
__device__ __forceinline__ void load8(const KT* __restrict__ p, KT v[8]) {
  if constexpr (sizeof(KT) == 4) {
    const float4* q = reinterpret_cast<const float4*>(p);
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      float4 t = __ldcg(q + i);
      v[4 * i] = t.x; v[4 * i + 1] = t.y; v[4 * i + 2] = t.z; v[4 * i + 3] = t.w;
    }
  } else {
    const double2* q = reinterpret_cast<const double2*>(p);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      double2 t = __ldcg(q + i);
      v[2 * i] = t.x; v[2 * i + 1] = t.y;
    }
  }
}

// Pair item: off-diagonal block and its transpose.
template <typename KT, int NPE>
__device__ __forceinline__ void gather_pair(const GatherArgs& g, int32_t p, const KT* __restrict__ krec,
                                            KT* __restrict__ k_out) {
  using L = RecLayout<NPE>;
  const int4 info = __ldg(reinterpret_cast<const int4*>(g.pair_info) + p);
  const int32_t s0 = __ldg(g.pair_ptr + p), s1 = __ldg(g.pair_ptr + p + 1);
  KT acc[9];
#pragma unroll
  for (int j = 0; j < 9; ++j) acc[j] = (KT)0;
  for (int32_t s = s0; s < s1; ++s) {
    const int32_t src = __ldg(g.pair_src + s);
    const int64_t e = src >> 6;
    const int slot = src & 63;
    KT v[12];
    load12<KT>(krec + (e & g.ring_mask) * L::kK + L::pair_off(slot), v);
#pragma unroll
    for (int j = 0; j < 9; ++j) acc[j] += v[j];
  }
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      k_out[info.x + (int64_t)info.y * k + m] = acc[3 * k + m];
      k_out[info.z + (int64_t)info.w * m + k] = acc[3 * k + m];
    }
}

// Node item: diagonal block and/or f.
template <typename KT, int NPE, bool WANT_K, bool WANT_F>
__device__ __forceinline__ void gather_node(const GatherArgs& g, int32_t n, const KT* __restrict__ krec,
                                            const double* __restrict__ frec, KT* __restrict__ k_out,
                                            double* __restrict__ f_out) {
  using L = RecLayout<NPE>;
  const int4 info = __ldg(reinterpret_cast<const int4*>(g.node_info) + n);
  const int32_t s0 = __ldg(g.node_ptr + n), s1 = __ldg(g.node_ptr + n + 1);
  KT acc[6];
#pragma unroll
  for (int j = 0; j < 6; ++j) acc[j] = (KT)0;
  double fa[3] = {0.0, 0.0, 0.0};
  for (int32_t s = s0; s < s1; ++s) {
    const int32_t src = __ldg(g.node_src + s);
    const int64_t e = src >> 4;
    const int a = src & 15;
    const int64_t slot = e & g.ring_mask;
    if constexpr (WANT_K) {
      KT v[8];
      load8<KT>(krec + slot * L::kK + L::diag_off(a), v);
#pragma unroll
      for (int j = 0; j < 6; ++j) acc[j] += v[j];
    }
    if constexpr (WANT_F) {
      const double* fp = frec + slot * L::kF + 3 * a;
      fa[0] += __ldcg(fp);
      fa[1] += __ldcg(fp + 1);
      fa[2] += __ldcg(fp + 2);
    }
  }
  if constexpr (WANT_K) {
    if (info.y > 0) {
      const KT full[9] = {acc[0], acc[1], acc[2], acc[1], acc[3], acc[4], acc[2], acc[4], acc[5]};
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int m = 0; m < 3; ++m) k_out[info.x + (int64_t)info.y * k + m] = full[3 * k + m];
    }
  }
  if constexpr (WANT_F) {
    f_out[3 * (int64_t)info.z + 0] = fa[0];
    f_out[3 * (int64_t)info.z + 1] = fa[1];
    f_out[3 * (int64_t)info.z + 2] = fa[2];
  }
}

// Store a 12-value off-diagonal block record (9 used), transposed when `swap`.
template <typename KT>
__device__ __forceinline__ void store_pair_block(KT* __restrict__ dst, const KT b[9], bool swap) {
  KT o[12];
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int m = 0; m < 3; ++m) o[3 * k + m] = swap ? b[3 * m + k] : b[3 * k + m];
  o[9] = o[10] = o[11] = (KT)0;
  if constexpr (sizeof(KT) == 4) {
    float4* q = reinterpret_cast<float4*>(dst);
#pragma unroll
    for (int i = 0; i < 3; ++i) __stcg(q + i, make_float4(o[4 * i], o[4 * i + 1], o[4 * i + 2], o[4 * i + 3]));
  } else {
    double2* q = reinterpret_cast<double2*>(dst);
#pragma unroll
    for (int i = 0; i < 6; ++i) __stcg(q + i, make_double2(o[2 * i], o[2 * i + 1]));
  }
}

// Store a diagonal block record: xx xy xz yy yz zz (+2 pad).
template <typename KT>
__device__ __forceinline__ void store_diag_block(KT* __restrict__ dst, const KT d[6]) {
  if constexpr (sizeof(KT) == 4) {
    float4* q = reinterpret_cast<float4*>(dst);
    __stcg(q, make_float4(d[0], d[1], d[2], d[3]));
    __stcg(q + 1, make_float4(d[4], d[5], 0.f, 0.f));
  } else {
    double2* q = reinterpret_cast<double2*>(dst);
    __stcg(q, make_double2(d[0], d[1]));
    __stcg(q + 1, make_double2(d[2], d[3]));
    __stcg(q + 2, make_double2(d[4], d[5]));
    __stcg(q + 3, make_double2(0.0, 0.0));
  }
}

}  // namespace psx
