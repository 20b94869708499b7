// Owner-computes gather of element records into the CSR values and f (kernel "B").
//
// The element phase writes, per element e, a record into a ring of scratch slots
// (slot = e & ring_mask):
//   K part (KT): npair off-diagonal 3x3 blocks, 12 values each (9 used, 16-byte
//                aligned), oriented with rows = the element node of smaller global id;
//                then npe diagonal blocks, 8 values each (xx xy xz yy yz zz + 2 pad).
//                npair = npe (npe - 1) / 2.
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
  // tile records (Tet4): lists name (tile, local pair / node).  A tile's ring slot holds,
  // with cap_p4 / cap_n4 = cap_p / cap_n rounded up to a multiple of 4, the planes
  // P0 (cap_p4 float4: pair values 0-3), P1 (float4: 4-7), P2 (cap_p4 floats: value 8),
  // D0 (cap_n4 float4: xx xy xz yy), D1 (cap_n4 float2: yz zz) in the K ring and
  // F0, F1, F2 (cap_n4 doubles: f x, y, z) in the f ring
  const int32_t* pair_ptr_t;
  const int32_t* pair_src_t;  // tile * 256 + local pair
  const int32_t* node_ptr_t;
  const int32_t* node_src_t;  // tile * 128 + local node
  int64_t ring_tile_mask;
  int32_t cap_p, cap_n;
  int32_t cap_p4, cap_n4;
  int32_t tile_k;             // K values per tile record: 9 cap_p4 + 6 cap_n4
  // per-tile reduction lists (psx_tile_plan_fill): one block of meta_stride bytes per
  // tile, fields at byte offsets off_n (node offsets), src_n (node codes), off_p (pair
  // offsets), src_p (pair codes); byte 0 / 1 = pair / node count.  The first
  // meta_node_bytes hold the count bytes and the node lists.
  const uint8_t* tile_meta;
  int32_t meta_stride, meta_node_bytes, off_p, off_n, src_p, src_n;
  int32_t tile;
};

// 16-byte vector loads/stores of record blocks (L2-only loads: the ring is rewritten while
// the kernel runs, so nothing may be served from a stale L1 line).
template <typename KT, int N>
__device__ __forceinline__ void load_block(const KT* __restrict__ p, KT v[N]) {
  if constexpr (sizeof(KT) == 4) {
    const float4* q = reinterpret_cast<const float4*>(p);
#pragma unroll
    for (int i = 0; i < N / 4; ++i) {
      const float4 t = __ldcg(q + i);
      v[4 * i] = t.x; v[4 * i + 1] = t.y; v[4 * i + 2] = t.z; v[4 * i + 3] = t.w;
    }
  } else {
    const double2* q = reinterpret_cast<const double2*>(p);
#pragma unroll
    for (int i = 0; i < N / 2; ++i) {
      const double2 t = __ldcg(q + i);
      v[2 * i] = t.x; v[2 * i + 1] = t.y;
    }
  }
}

// GLOBAL: `p` is global memory (L2-only store); otherwise a plain store through a
// generic pointer (used for the shared-memory staging of records).
template <typename KT, int N, bool GLOBAL = true>
__device__ __forceinline__ void store_block(KT* __restrict__ p, const KT v[N]) {
  if constexpr (!GLOBAL && sizeof(KT) == 4) {
    // shared-memory staging: 16-byte stores (a record stride of 108 floats keeps the
    // 8 lanes of each store phase on distinct banks)
    float4* q = reinterpret_cast<float4*>(p);
#pragma unroll
    for (int i = 0; i < N / 4; ++i) q[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
  } else if constexpr (!GLOBAL) {
#pragma unroll
    for (int i = 0; i < N; ++i) p[i] = v[i];
  } else if constexpr (sizeof(KT) == 4) {
    float4* q = reinterpret_cast<float4*>(p);
#pragma unroll
    for (int i = 0; i < N / 4; ++i) st_ring(q + i, make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]));
  } else {
    double2* q = reinterpret_cast<double2*>(p);
#pragma unroll
    for (int i = 0; i < N / 2; ++i) st_ring(q + i, make_double2(v[2 * i], v[2 * i + 1]));
  }
}

// Tet4 element records in the global ring are stored in planes: the 16-byte granule i of
// the record of ring slot s lies at krec + (i * plane + s) * W (W = 16 / sizeof(KT) values,
// plane = ring length), so that the 32 lanes of a warp, which write consecutive slots,
// write whole sectors.  `base` = krec + s * W; `o` = value offset inside the record
// (RecLayout<4>, a multiple of W).
template <typename KT, int N>
__device__ __forceinline__ void store_planes(KT* __restrict__ base, int o, const KT v[N], int64_t plane) {
  constexpr int W = 16 / (int)sizeof(KT);
#pragma unroll
  for (int i = 0; i < N / W; ++i) {
    KT* q = base + (int64_t)(o / W + i) * plane * W;
    if constexpr (W == 4)
      st_ring(reinterpret_cast<float4*>(q), make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]));
    else
      st_ring(reinterpret_cast<double2*>(q), make_double2(v[2 * i], v[2 * i + 1]));
  }
}
template <typename KT, int N>
__device__ __forceinline__ void load_planes(const KT* __restrict__ base, int o, KT v[N], int64_t plane) {
  constexpr int W = 16 / (int)sizeof(KT);
#pragma unroll
  for (int i = 0; i < N / W; ++i) {
    const KT* q = base + (int64_t)(o / W + i) * plane * W;
    if constexpr (W == 4) {
      const float4 t = __ldcg(reinterpret_cast<const float4*>(q));
      v[4 * i] = t.x; v[4 * i + 1] = t.y; v[4 * i + 2] = t.z; v[4 * i + 3] = t.w;
    } else {
      const double2 t = __ldcg(reinterpret_cast<const double2*>(q));
      v[2 * i] = t.x; v[2 * i + 1] = t.y;
    }
  }
}

// Contributions whose loads are issued together, kept within the register budget: the
// fused FP32 f + K Tet4 kernel runs 3 blocks per SM, which its 168 registers allow only
// with two pair and one node contribution in flight; the other sweeps keep four.
template <typename KT, int NPE, bool WANT_K, bool WANT_F>
struct PairBatch {
  static constexpr int n = sizeof(KT) == 8 ? 2 : (NPE == 4 && WANT_K && WANT_F ? 2 : 4);
};
template <typename KT, int NPE, bool WANT_K, bool WANT_F>
struct NodeBatch {
  static constexpr int n = sizeof(KT) == 8 ? 2 : (NPE == 4 && WANT_K && WANT_F ? 1 : 4);
};

// What a gather item starts from: its output positions (pair_info / node_info) and the
// bounds of its contribution list.  The warp-specialised gather loads it for its next
// task while the current one runs.
struct ItemHead {
  int4 info;
  int32_t s0, s1;
};
template <bool TILES>
__device__ __forceinline__ ItemHead pair_head(const GatherArgs& g, int32_t p) {
  const int32_t* lptr = TILES ? g.pair_ptr_t : g.pair_ptr;
  return ItemHead{__ldg(reinterpret_cast<const int4*>(g.pair_info) + p), __ldg(lptr + p), __ldg(lptr + p + 1)};
}
template <bool TILES>
__device__ __forceinline__ ItemHead node_head(const GatherArgs& g, int32_t n) {
  const int32_t* lptr = TILES ? g.node_ptr_t : g.node_ptr;
  return ItemHead{__ldg(reinterpret_cast<const int4*>(g.node_info) + n), __ldg(lptr + n), __ldg(lptr + n + 1)};
}

// Pair item: off-diagonal block and its transpose.  Contributions are summed in list
// (ascending element) order; their loads are issued kBatch at a time.
template <typename KT, int NPE, bool TILES = false, bool WANT_F = false, int BATCH = 0, bool VSTORE = false>
__device__ __forceinline__ void gather_pair(const GatherArgs& g, const ItemHead& h, const KT* __restrict__ krec,
                                            KT* __restrict__ k_out) {
  using L = RecLayout<NPE>;
  const int4 info = h.info;
  const int32_t* list = TILES ? g.pair_src_t : g.pair_src;
  const int32_t s0 = h.s0, s1 = h.s1;
  KT acc[9];
#pragma unroll
  for (int j = 0; j < 9; ++j) acc[j] = (KT)0;
  constexpr int kBatch = BATCH > 0 ? BATCH : PairBatch<KT, NPE, true, WANT_F>::n;
  for (int32_t s = s0; s < s1; s += kBatch) {
    int32_t src[kBatch];
#pragma unroll
    for (int b = 0; b < kBatch; ++b) src[b] = (s + b < s1) ? __ldg(list + s + b) : -1;
    KT v[kBatch][12];
#pragma unroll
    for (int b = 0; b < kBatch; ++b)
      if (src[b] >= 0) {
        if constexpr (TILES) {
          // pair planes of the tile record (K is FP32 wherever tile records hold K)
          const float* base = reinterpret_cast<const float*>(krec) + ((int64_t)(src[b] >> 8) & g.ring_tile_mask) * g.tile_k;
          const int lp = src[b] & 255;
          const float4 x = __ldcg(reinterpret_cast<const float4*>(base) + lp);
          const float4 y = __ldcg(reinterpret_cast<const float4*>(base + 4 * g.cap_p4) + lp);
          v[b][0] = x.x; v[b][1] = x.y; v[b][2] = x.z; v[b][3] = x.w;
          v[b][4] = y.x; v[b][5] = y.y; v[b][6] = y.z; v[b][7] = y.w;
          v[b][8] = __ldcg(base + 8 * g.cap_p4 + lp);
        } else if constexpr (NPE == 4) {
          constexpr int W = 16 / (int)sizeof(KT);
          load_planes<KT, 12>(krec + ((int64_t)(src[b] >> 6) & g.ring_mask) * W, L::pair_off(src[b] & 63), v[b],
                              g.ring_mask + 1);
        } else {
          load_block<KT, 12>(krec + ((int64_t)(src[b] >> 6) & g.ring_mask) * L::kK + L::pair_off(src[b] & 63), v[b]);
        }
      }
#pragma unroll
    for (int b = 0; b < kBatch; ++b)
      if (src[b] >= 0) {
#pragma unroll
        for (int j = 0; j < 9; ++j) acc[j] += v[b][j];
      }
  }
  if constexpr (VSTORE) {
#pragma unroll
    for (int k = 0; k < 3; ++k) store3(k_out + info.x + (int64_t)info.y * k, acc[3 * k], acc[3 * k + 1], acc[3 * k + 2]);
#pragma unroll
    for (int m = 0; m < 3; ++m) store3(k_out + info.z + (int64_t)info.w * m, acc[m], acc[3 + m], acc[6 + m]);
  } else {
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int m = 0; m < 3; ++m) {
        __stcs(k_out + info.x + (int64_t)info.y * k + m, acc[3 * k + m]);
        __stcs(k_out + info.z + (int64_t)info.w * m + k, acc[3 * k + m]);
      }
  }
}

// Dynamic-relaxation epilogue of a node item (the viscous update of
// psierra analysis/dynamic_relaxation.py:296-299, 378-382 on the linearised system).
struct DRArgs {
  const double* b;
  const double* minv;
  double c1, c2, dt;
  double* x;
  double* vel;
};

// Node item: diagonal block and/or f (or, with DR, the fused pseudo-step on f = K x).
template <typename KT, int NPE, bool WANT_K, bool WANT_F, bool DR = false, bool TILES = false, int BATCH = 0,
          bool VSTORE = false>
__device__ __forceinline__ void gather_node(const GatherArgs& g, const ItemHead& h, const KT* __restrict__ krec,
                                            const double* __restrict__ frec, KT* __restrict__ k_out,
                                            double* __restrict__ f_out, const DRArgs* dr = nullptr) {
  using L = RecLayout<NPE>;
  const int4 info = h.info;
  const int32_t* list = TILES ? g.node_src_t : g.node_src;
  const int32_t s0 = h.s0, s1 = h.s1;
  KT acc[6];
#pragma unroll
  for (int j = 0; j < 6; ++j) acc[j] = (KT)0;
  double fa[3] = {0.0, 0.0, 0.0};
  constexpr int kBatch = BATCH > 0 ? BATCH : NodeBatch<KT, NPE, WANT_K, WANT_F>::n;
  for (int32_t s = s0; s < s1; s += kBatch) {
    int32_t src[kBatch];
#pragma unroll
    for (int b = 0; b < kBatch; ++b) src[b] = (s + b < s1) ? __ldg(list + s + b) : -1;
    KT v[kBatch][8];
    double fv[kBatch][3];
#pragma unroll
    for (int b = 0; b < kBatch; ++b)
      if (src[b] >= 0) {
        if constexpr (TILES) {
          // diagonal and f planes of the tile record (K is FP32 wherever it is present)
          const int64_t slot = (int64_t)(src[b] >> 7) & g.ring_tile_mask;
          const int ln = src[b] & 127;
          if constexpr (WANT_K) {
            const float* base = reinterpret_cast<const float*>(krec) + slot * g.tile_k + 9 * g.cap_p4;
            const float4 x = __ldcg(reinterpret_cast<const float4*>(base) + ln);
            const float2 y = __ldcg(reinterpret_cast<const float2*>(base + 4 * g.cap_n4) + ln);
            v[b][0] = x.x; v[b][1] = x.y; v[b][2] = x.z; v[b][3] = x.w;
            v[b][4] = y.x; v[b][5] = y.y;
          }
          if constexpr (WANT_F) {
            const double* fb = frec + slot * 3 * g.cap_n4 + ln;
            fv[b][0] = __ldcg(fb);
            fv[b][1] = __ldcg(fb + g.cap_n4);
            fv[b][2] = __ldcg(fb + 2 * g.cap_n4);
          }
        } else if constexpr (NPE == 4) {
          // planar Tet4 element records (store_planes); f: value j of the 12 at granule j/2
          constexpr int W = 16 / (int)sizeof(KT);
          const int64_t slot = (int64_t)(src[b] >> 4) & g.ring_mask;
          const int64_t plane = g.ring_mask + 1;
          const int a = src[b] & 15;
          if constexpr (WANT_K) load_planes<KT, 8>(krec + slot * W, L::diag_off(a), v[b], plane);
          if constexpr (WANT_F) {
#pragma unroll
            for (int j = 0; j < 3; ++j) {
              const int vj = 3 * a + j;
              fv[b][j] = __ldcg(frec + slot * 2 + (int64_t)(vj >> 1) * plane * 2 + (vj & 1));
            }
          }
        } else {
          const int64_t slot = (int64_t)(src[b] >> 4) & g.ring_mask;
          const int a = src[b] & 15;
          const KT* kp = krec + slot * L::kK + L::diag_off(a);
          const double* fp = frec + slot * L::kF + 3 * a;
          if constexpr (WANT_K) load_block<KT, 8>(kp, v[b]);
          if constexpr (WANT_F) {
            fv[b][0] = __ldcg(fp);
            fv[b][1] = __ldcg(fp + 1);
            fv[b][2] = __ldcg(fp + 2);
          }
        }
      }
#pragma unroll
    for (int b = 0; b < kBatch; ++b)
      if (src[b] >= 0) {
        if constexpr (WANT_K) {
#pragma unroll
          for (int j = 0; j < 6; ++j) acc[j] += v[b][j];
        }
        if constexpr (WANT_F) {
          fa[0] += fv[b][0];
          fa[1] += fv[b][1];
          fa[2] += fv[b][2];
        }
      }
  }
  if constexpr (WANT_K) {
    if (info.y > 0) {
      const KT full[9] = {acc[0], acc[1], acc[2], acc[1], acc[3], acc[4], acc[2], acc[4], acc[5]};
      if constexpr (VSTORE) {
#pragma unroll
        for (int k = 0; k < 3; ++k)
          store3(k_out + info.x + (int64_t)info.y * k, full[3 * k], full[3 * k + 1], full[3 * k + 2]);
      } else {
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
          for (int m = 0; m < 3; ++m) __stcs(k_out + info.x + (int64_t)info.y * k + m, full[3 * k + m]);
      }
    }
  }
  if constexpr (DR) {
    // every element reading x_i has been evaluated (they are this item's contributions)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const int64_t d = 3 * (int64_t)info.z + k;
      const double r = dr->b[d] - fa[k];
      const double a = dr->minv[d] * r;
      const double v = dr->c1 * dr->vel[d] + dr->c2 * a;
      dr->vel[d] = v;
      dr->x[d] += dr->dt * v;
      if (f_out) f_out[d] = r;
    }
  } else if constexpr (WANT_F) {
    __stcs(f_out + 3 * (int64_t)info.z + 0, fa[0]);
    __stcs(f_out + 3 * (int64_t)info.z + 1, fa[1]);
    __stcs(f_out + 3 * (int64_t)info.z + 2, fa[2]);
  }
}

// Store an off-diagonal block record (9 values + 3 pad), transposed when `swap`.
template <typename KT, bool GLOBAL = true>
__device__ __forceinline__ void store_pair_block(KT* __restrict__ dst, const KT b[9], bool swap) {
  KT o[12];
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int m = 0; m < 3; ++m) o[3 * k + m] = swap ? b[3 * m + k] : b[3 * k + m];
  o[9] = o[10] = o[11] = (KT)0;
  store_block<KT, 12, GLOBAL>(dst, o);
}

// Store a diagonal block record: xx xy xz yy yz zz (+2 pad).
template <typename KT, bool GLOBAL = true>
__device__ __forceinline__ void store_diag_block(KT* __restrict__ dst, const KT d[6]) {
  const KT o[8] = {d[0], d[1], d[2], d[3], d[4], d[5], (KT)0, (KT)0};
  store_block<KT, 8, GLOBAL>(dst, o);
}

// ---- persistent task queue --------------------------------------------------------
// Tasks are claimed by warps (32 elements or 32 items each).  Counters live at the
// start of the workspace: [0] next task, [1 .. G] element tiles finished per granule,
// [1 + G .. 2G] gather tiles finished per granule, [1 + 2G] next gather task of the
// warp-specialised kernel (whose [0] counts element tiles).
struct QueueArgs {
  const int4* tasks;
  int32_t n_tasks;
  int32_t n_granules;
  const int32_t* btiles;  // gather tiles per granule
  int32_t* counters;
  int32_t granule_log2;
  int32_t tile;
  int32_t span_g;         // max item span in granules (rounded up)
  int32_t ring_g;         // ring length in granules (power of two)
  int64_t n_elements;
  int32_t max_spins;      // polls of one bounded wait before it gives up
};

constexpr int32_t kDefaultWaitSpins = 1 << 22;  // about a second with the 200 ns back-off

// Count one finished element tile: a release add, so the tile's record writes (those
// of every lane: the caller's __syncwarp orders them before lane 0's release) are
// visible to a gather that acquires the count.  Used by the warp-specialised kernel
// (K-only 0.72 -> 0.69 ms on the 3.07M-element cube); the mixed kernel keeps a fence
// and a plain add, which measured faster there (FP64 K.v 0.36 vs 0.33 ms with the
// release add).
__device__ __forceinline__ void publish_tile(int32_t* p) {
  asm volatile("red.release.gpu.global.add.s32 [%0], 1;" ::"l"(p) : "memory");
}

__device__ __forceinline__ int32_t ld_acquire(const int32_t* p) {
  int32_t v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Bounded wait, executed by a whole warp: lane j checks counter[first + j] >=
// target(first + j) for j < count.  Returns false (and flags the status) if the wait
// gives up; the caller then still proceeds, so every access stays in bounds and the
// host reports the failure.
template <typename Target>
__device__ __forceinline__ bool wait_counters(const int32_t* cnt, int32_t first, int32_t count, Target target,
                                              Status* st, int32_t max_spins) {
  const int lane = threadIdx.x & 31;
  for (int32_t base = 0; base < count; base += 32) {
    const int32_t g = first + base + lane;
    const bool mine = (base + lane) < count && g >= 0;
    const int32_t want = mine ? target(g) : 0;
    int spins = 0;
    while (true) {
      const bool ok = !mine || ld_acquire(cnt + g) >= want;
      if (__all_sync(0xffffffffu, ok)) break;
      // once any wait has given up, every later wait returns at once
      if (++spins > max_spins || (ld_acquire(&st->flags) & 1)) {
        if (lane == 0) atomicOr(&st->flags, 1);
        return false;
      }
      if (spins > 64) __nanosleep(200);
    }
    if (spins && lane == 0) atomicAdd(&st->iters, spins);
  }
  return true;
}

// Bounded wait on a prefix, executed by a whole warp: returns once every granule
// g <= need has reached target(g).  `done` is the warp's watermark (every granule
// <= done is known complete; start at -1): a wait below it costs nothing, and each poll
// reads the 32 counters after it in one load and advances it over their complete run,
// so one poll usually covers the warp's next few tasks.  A prefix implies the spans the
// queue needs (an element tile: the gathers of the granules its ring slots held; a
// gather: the element tiles of its span), and everything it adds was claimed earlier in
// the same in-order lists, so the queue still drains.  After `max_spins` polls (or
// once another wait has given up) it sets status flag bit 0 and returns false; the
// caller still proceeds, so every access stays in bounds and the host reports it.
template <typename Target>
__device__ __forceinline__ bool wait_prefix(const int32_t* cnt, int32_t need, int32_t n, Target target, int32_t& done,
                                            Status* st, int32_t max_spins) {
  if (need <= done) return true;
  const int lane = threadIdx.x & 31;
  int spins = 0;
  while (true) {
    const int32_t g = done + 1 + lane;
    const bool ok = g >= n || ld_acquire(cnt + g) >= target(g);
    const unsigned m = __ballot_sync(0xffffffffu, ok);
    done += m == 0xffffffffu ? 32 : __ffs(~m) - 1;
    if (need <= done) break;
    if (++spins > max_spins || (ld_acquire(&st->flags) & 1)) {
      if (lane == 0) atomicOr(&st->flags, 1);
      return false;
    }
    if (spins > 64) __nanosleep(200);
  }
  if (spins && lane == 0) atomicAdd(&st->iters, spins);
  return true;
}


// ---- persistent queue loop -----------------------------------------------------------
// Each warp claims tasks in queue order (the claim of the next task is issued before the
// current one is worked on).  Element tiles wait until the gather tiles still reading
// the ring slots they overwrite are done, run `element_tile(task)` and publish their
// granule; gather tiles wait for the element granules they read and sum them.  Every
// wait is on a task earlier in the queue (psx_task_fill), so the queue always drains.
template <typename KT, int NPE, bool WANT_K, bool WANT_F, bool DR, bool TILES, typename ElementTile>
__device__ __forceinline__ void drain_queue(const GatherArgs& g, const QueueArgs& Q, Status* st,
                                            const KT* __restrict__ krec, const double* __restrict__ frec,
                                            KT* __restrict__ k_out, double* __restrict__ f_out, const DRArgs& dr,
                                            ElementTile&& element_tile) {
  const int lane = threadIdx.x & 31;
  int32_t* acnt = Q.counters + 1;
  int32_t* bcnt = Q.counters + 1 + Q.n_granules;
  const int64_t gsize = (int64_t)1 << Q.granule_log2;
  auto atiles = [&](int32_t r) -> int32_t {
    const int64_t n = min(gsize, Q.n_elements - (int64_t)r * gsize);
    return (int32_t)((n + Q.tile - 1) / Q.tile);
  };
  auto btiles = [&](int32_t r) -> int32_t { return __ldg(Q.btiles + r); };
  // this loop keeps the span waits: prefix waits (wait_prefix, as in the split kernel's
  // loops) measured slower here, where one warp runs both kinds of task (K.v 0.298 ->
  // 0.351 ms, f only 0.284 -> 0.350 ms on the 80^3 cube)
  int32_t next = 0;
  if (lane == 0) next = atomicAdd(Q.counters, 1);
  while (true) {
    const int32_t t = __shfl_sync(0xffffffffu, next, 0);
    if (t >= Q.n_tasks) break;
    if (lane == 0) next = atomicAdd(Q.counters, 1);
    const int4 task = __ldg(Q.tasks + t);
    const int32_t gr = task.y;
    if (task.x == 0) {
      const int32_t old = gr - Q.ring_g;  // granule whose ring slots this tile overwrites
      if (old >= 0) wait_counters(bcnt, old, min(Q.span_g + 2, Q.n_granules - old), btiles, st, Q.max_spins);
      __syncwarp();
      element_tile(task);
      __syncwarp();
      if (lane == 0) {
        __threadfence();
        atomicAdd(acnt + gr, 1);
      }
    } else {
      const int32_t first = max(0, gr - Q.span_g - 1);
      wait_counters(acnt, first, gr - first + 1, atiles, st, Q.max_spins);
      __syncwarp();
      for (int32_t item = task.z + lane; item < task.w; item += 32) {
        // K row segments leave as vector + scalar pairs (FP64 f+K 2.35 -> 2.26 ms, Tet10
        // 0.70 / 1.10 -> 0.66 / 1.05 ms on the benchmark meshes)
        if (task.x == 1) {
          if constexpr (WANT_K) gather_pair<KT, NPE, TILES, WANT_F, 0, true>(g, pair_head<TILES>(g, item), krec, k_out);
        } else {
          gather_node<KT, NPE, WANT_K, WANT_F, DR, TILES, 0, true>(g, node_head<TILES>(g, item), krec, frec, k_out,
                                                                    f_out, &dr);
        }
      }
      __syncwarp();
      if (lane == 0) atomicAdd(bcnt + gr, 1);
    }
  }
}

// ---- warp-specialised queue loops -----------------------------------------------------
// The split kernel runs element tiles and gathers in different warps.  Element tiles are
// claimed in index order from counter `ecnt` (tile i = elements [i tile, (i+1) tile)),
// gather tiles in list order from `gcnt` over the gather tasks of the K queue.  The waits
// are those of drain_queue: an element tile waits for the gathers still reading the ring
// slots it overwrites, a gather tile for the element tiles of its granule span.  Every
// task waits only on tasks claimed before it (claims are in order in both lists), so the
// loops cannot deadlock while the warps that claimed tasks are resident; a wait that
// gives up flags the status and the task proceeds in bounds.
// Tuning switches of the warp-specialised loops: load the next element tile's
// connectivity / the next gather task's item heads while the current one runs.  On the
// 80^3 cube (f+K) the connectivity prefetch is neutral (0.616-0.619 against
// 0.616-0.621 ms); the head prefetch spills at 80 gather registers and, with the
// 160 / 96 split it needs, ran 0.643 ms.
#ifndef PSX_SPLIT_PREFETCH_CONN
#define PSX_SPLIT_PREFETCH_CONN 1
#endif
#ifndef PSX_SPLIT_PREFETCH_HEADS
#define PSX_SPLIT_PREFETCH_HEADS 0
#endif

template <typename ElementTile>
__device__ __forceinline__ void drain_elements(const QueueArgs& Q, const int4* __restrict__ conn, int32_t* ecnt,
                                               Status* st, ElementTile&& element_tile) {
  const int lane = threadIdx.x & 31;
  int32_t* acnt = Q.counters + 1;
  int32_t* bcnt = Q.counters + 1 + Q.n_granules;
  auto btiles = [&](int32_t r) -> int32_t { return __ldg(Q.btiles + r); };
  const int64_t n_tiles = (Q.n_elements + Q.tile - 1) / Q.tile;
  int32_t gathered = -1;  // watermark: the gathers of every granule <= gathered are done
  // A finished tile is published during the warp's next tile, after that tile's
  // evaluation: the release then finds the tile's record stores long completed instead
  // of waiting for them (relaxed adds in place of the release measured 9% faster).  The
  // warp publishes before any wait that could block, so it never waits while holding an
  // unpublished tile and the queue drains as before.
  int32_t pending = -1;
  auto publish_pending = [&]() {
    if (pending >= 0 && lane == 0) publish_tile(acnt + pending);
    pending = -1;
  };
  // Tiles are claimed two ahead, so that the next tile's connectivity is loaded while
  // the current one is evaluated (its node loads then start one memory round trip
  // earlier).  A claimed tile waits only on earlier work, like every other task.
  auto conn_of = [&](int32_t t) -> int4 {
    const int64_t e = (int64_t)t * Q.tile + lane;
    return (t < n_tiles && e < Q.n_elements) ? __ldg(conn + e) : make_int4(0, 0, 0, 0);
  };
  constexpr bool kPre = PSX_SPLIT_PREFETCH_CONN != 0;
  int32_t claim = 0;
  if (lane == 0) claim = atomicAdd(ecnt, 1);
  int32_t t = __shfl_sync(0xffffffffu, claim, 0);
  if (lane == 0 && t < n_tiles) claim = atomicAdd(ecnt, 1);
  int4 cn = kPre ? conn_of(t) : make_int4(0, 0, 0, 0);
  while (t < n_tiles) {
    const int32_t tn = __shfl_sync(0xffffffffu, claim, 0);
    if (lane == 0 && tn < n_tiles) claim = atomicAdd(ecnt, 1);
    const int4 cn_next = kPre ? conn_of(tn) : make_int4(0, 0, 0, 0);
    if constexpr (!kPre) cn = conn_of(t);
    const int64_t e0 = (int64_t)t * Q.tile;
    const int64_t e1 = min(e0 + (int64_t)Q.tile, Q.n_elements);
    const int32_t gr = (int32_t)(e0 >> Q.granule_log2);
    const int32_t old = gr - Q.ring_g;  // granule whose ring slots this tile overwrites
    if (old >= 0) {
      const int32_t need = min(old + Q.span_g + 1, Q.n_granules - 1);
      if (need > gathered) publish_pending();
      wait_prefix(bcnt, need, Q.n_granules, btiles, gathered, st, Q.max_spins);
    }
    __syncwarp();
    element_tile(make_int4(0, gr, (int32_t)e0, (int32_t)e1), cn, publish_pending);
    __syncwarp();
    publish_pending();  // no-op unless the tile did not publish its predecessor
    pending = gr;
    t = tn;
    cn = cn_next;
  }
  __syncwarp();
  publish_pending();
}

template <typename KT, int NPE, bool WANT_K, bool WANT_F, int PAIR_BATCH, int NODE_BATCH>
__device__ __forceinline__ void drain_gathers(const GatherArgs& g, const QueueArgs& Q, const int4* __restrict__ gtasks,
                                              int32_t n_gtasks, int32_t* gcnt, Status* st,
                                              const KT* __restrict__ krec, const double* __restrict__ frec,
                                              KT* __restrict__ k_out, double* __restrict__ f_out) {
  const int lane = threadIdx.x & 31;
  int32_t* acnt = Q.counters + 1;
  int32_t* bcnt = Q.counters + 1 + Q.n_granules;
  const int64_t gsize = (int64_t)1 << Q.granule_log2;
  auto atiles = [&](int32_t r) -> int32_t {
    const int64_t n = min(gsize, Q.n_elements - (int64_t)r * gsize);
    return (int32_t)((n + Q.tile - 1) / Q.tile);
  };
  int32_t evaluated = -1;  // watermark: the element tiles of every granule <= evaluated are done
  // Tasks are claimed two ahead: the next task and the heads of its items (output
  // positions and list bounds, plan data that no wait guards) are loaded while the
  // current task runs, which takes one memory round trip off each task's chain.
  constexpr bool kPre = PSX_SPLIT_PREFETCH_HEADS != 0;
  auto head_of = [&](const int4& task) -> ItemHead {
    const int32_t item = task.z + lane;
    if (item >= task.w) return ItemHead{make_int4(0, 0, 0, 0), 0, 0};
    return task.x == 1 ? pair_head<true>(g, item) : node_head<true>(g, item);
  };
  int32_t claim = 0;
  if (lane == 0) claim = atomicAdd(gcnt, 1);
  int32_t t = __shfl_sync(0xffffffffu, claim, 0);
  if (lane == 0 && t < n_gtasks) claim = atomicAdd(gcnt, 1);
  int4 task = make_int4(0, 0, 0, 0);
  ItemHead head{make_int4(0, 0, 0, 0), 0, 0};
  if (t < n_gtasks) {
    task = __ldg(gtasks + t);
    if constexpr (kPre) head = head_of(task);
  }
  while (t < n_gtasks) {
    const int32_t tn = __shfl_sync(0xffffffffu, claim, 0);
    if (lane == 0 && tn < n_gtasks) claim = atomicAdd(gcnt, 1);
    int4 task_n = make_int4(0, 0, 0, 0);
    ItemHead head_n{make_int4(0, 0, 0, 0), 0, 0};
    if (tn < n_gtasks) {
      task_n = __ldg(gtasks + tn);
      if constexpr (kPre) head_n = head_of(task_n);
    }
    const int32_t gr = task.y;
    wait_prefix(acnt, gr, Q.n_granules, atiles, evaluated, st, Q.max_spins);
    __syncwarp();
    // K values leave in float2 + float pairs per row segment: 12 instead of 18 store
    // instructions per pair block (f+K 0.76 -> 0.72 ms, K-only 0.69 -> 0.64 ms on the
    // 3.07M-element cube; the memory pipeline the two roles share is the bottleneck)
    for (int32_t item = task.z + lane; item < task.w; item += 32) {
      // a task's first 32 items use the preloaded heads
      const bool pre = kPre && item < task.z + 32;
      if (task.x == 1) {
        if constexpr (WANT_K)
          gather_pair<KT, NPE, true, WANT_F, PAIR_BATCH, true>(g, pre ? head : pair_head<true>(g, item), krec, k_out);
      } else {
        gather_node<KT, NPE, WANT_K, WANT_F, false, true, NODE_BATCH, true>(
            g, pre ? head : node_head<true>(g, item), krec, frec, k_out, f_out);
      }
    }
    __syncwarp();
    if (lane == 0) atomicAdd(bcnt + gr, 1);
    t = tn;
    task = task_n;
    head = head_n;
  }
}

inline GatherArgs gather_args(const psx_plan_t* P, int64_t ring_elems) {
  GatherArgs g;
  g.pair_info = P->pair_info;
  g.pair_ptr = P->pair_ptr;
  g.pair_src = P->pair_src;
  g.node_info = P->node_info;
  g.node_ptr = P->node_ptr;
  g.node_src = P->node_src;
  g.p0 = g.p1 = g.n0 = g.n1 = 0;
  g.ring_mask = ring_elems - 1;
  g.pair_ptr_t = P->pair_ptr_t;
  g.pair_src_t = P->pair_src_t;
  g.node_ptr_t = P->node_ptr_t;
  g.node_src_t = P->node_src_t;
  g.cap_p = P->tile_cap_pairs;
  g.cap_n = P->tile_cap_nodes;
  g.cap_p4 = (g.cap_p + 3) / 4 * 4;  // every plane starts on a 16-byte boundary
  g.cap_n4 = (g.cap_n + 3) / 4 * 4;
  g.tile_k = 9 * g.cap_p4 + 6 * g.cap_n4;
  g.tile_meta = P->tile_meta;
  g.tile = P->tile;
  {
    const int32_t T = P->tile > 0 ? P->tile : 1;
    auto up4 = [](int32_t b) { return (b + 3) / 4 * 4; };
    g.off_n = 4;
    g.src_n = g.off_n + up4(4 * T + 1);
    g.off_p = g.src_n + 4 * T;
    g.src_p = g.off_p + up4(6 * T + 1);
    g.meta_stride = (g.src_p + 6 * T + 15) / 16 * 16;
    g.meta_node_bytes = (g.off_p + 15) / 16 * 16;  // header and node lists
  }
  g.ring_tile_mask = P->tile > 0 ? ring_elems / P->tile - 1 : 0;
  return g;
}

// ---- workspace layout (host side) ---------------------------------------------------
struct WorkLayout {
  int32_t* counters;
  size_t counter_bytes;
  void* krec;
  double* frec;
  int64_t ring_elems;
  int32_t ring_g;
  int32_t span_g;
  int32_t granule_log2;
  int32_t grid;
  int64_t total_bytes;
  bool tiles;  // tile records (Tet4, FP32 tangent or no tangent)
};

inline int32_t device_sm_count() {
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  return sms;
}

// Workspace of one assembly call: task counters, then the ring of K records (the K queue
// only), then the ring of f records (each 256-byte aligned).  The ring spans a
// power-of-two number of granules covering the item span, the queue's lag and the
// slack for tiles in flight; with `work` null only the sizes are computed.
inline int work_layout(const psx_plan_t* P, int precision, void* work, WorkLayout* W, int blocks_per_sm = 3,
                       bool queue_k = true) {
  if (!P || !W || P->n_elements <= 0 || P->n_nodes <= 0 || P->granule <= 0 || (P->granule & (P->granule - 1)))
    return PSX_ERR_ARG;
  if (!P->conn || !P->pair_info || !P->pair_ptr || !P->pair_src || !P->node_info || !P->node_ptr ||
      !P->node_src || !P->tasks_k || !P->tasks_f || !P->btiles_k || !P->btiles_f || P->tile <= 0)
    return PSX_ERR_ARG;
  if (precision != PSX_FP64 && precision != PSX_FP32_MIXED) return PSX_ERR_ARG;
  if (P->npe != 4 && P->npe != 10) return PSX_ERR_ARG;
  // Tet4 sweeps with an FP32 tangent or without a tangent sum shared blocks per element
  // tile (tile records); the FP64 tangent and Tet10 keep one record per element
  W->tiles = P->npe == 4 && (precision == PSX_FP32_MIXED || !queue_k);
  if (W->tiles) {
    if (!P->tile_meta || !P->pair_ptr_t || !P->pair_src_t || !P->node_ptr_t || !P->node_src_t || P->tile_cap_nodes <= 0 ||
        P->tile_cap_pairs < 0 || P->tile_cap_pairs > 192 || P->tile_cap_nodes > 128 || P->tile > 32 ||
        (P->tile & (P->tile - 1)) || P->granule % P->tile)
      return PSX_ERR_ARG;
  }
  const int kt = precision == PSX_FP64 ? 8 : 4;
  const int kK = P->npe == 4 ? RecLayout<4>::kK : RecLayout<10>::kK;
  const int kF = P->npe == 4 ? RecLayout<4>::kF : RecLayout<10>::kF;
  int32_t lg = 0;
  while (((int64_t)1 << lg) < P->granule) ++lg;
  W->granule_log2 = lg;
  W->span_g = (int32_t)((P->max_span + P->granule - 1) / P->granule);
  int32_t all = 1;
  while (all < P->n_granules) all <<= 1;
  // element tiles overwrite ring slots only after the gathers reading them are done; the
  // slack beyond span + lag is room for the element tiles in flight (at least 6 granules)
  const int32_t slack = P->ring_slack > 6 ? P->ring_slack : 6;
  int32_t ring = 1;
  const int32_t lag = queue_k || P->lag_f <= 0 ? P->lag : P->lag_f;
  while (ring < W->span_g + lag + slack) ring <<= 1;
  W->ring_g = ring < all ? ring : all;
  W->ring_elems = (int64_t)W->ring_g * P->granule;
  const int sms = device_sm_count();
  if (sms <= 0) return PSX_ERR_CUDA;
  const int64_t ntask = P->n_tasks_k > P->n_tasks_f ? P->n_tasks_k : P->n_tasks_f;
  // a plan may override the blocks per SM (the autotuner's knob); tasks are claimed in
  // queue order, so any grid is deadlock-free and extra blocks only queue for an SM
  const int bps = P->blocks_per_sm > 0 ? (P->blocks_per_sm < 4 ? P->blocks_per_sm : 4) : blocks_per_sm;
  W->grid = (int32_t)(sms * bps < ntask ? sms * bps : ntask);
  auto up = [](int64_t b) { return (b + 255) / 256 * 256; };
  // [0] next task (next element tile in the split kernel), [1, 1 + G) element tiles done
  // per granule, [1 + G, 1 + 2G) gather tiles done, [1 + 2G] next gather task (split)
  W->counter_bytes = (size_t)up(4 * (2 + 2 * (int64_t)P->n_granules));
  int64_t kbytes, fbytes;
  if (W->tiles) {
    const int64_t ring_tiles = W->ring_elems / P->tile;
    // planar tile records (GatherArgs): 9 cap_p4 + 6 cap_n4 K values, 3 cap_n4 f doubles
    const int64_t cp4 = (P->tile_cap_pairs + 3) / 4 * 4, cn4 = (P->tile_cap_nodes + 3) / 4 * 4;
    kbytes = queue_k ? up(ring_tiles * (9 * cp4 + 6 * cn4) * kt) : 0;
    fbytes = up(ring_tiles * 3 * cn4 * 8);
  } else {
    kbytes = queue_k ? up(W->ring_elems * kK * kt) : 0;
    fbytes = up(W->ring_elems * kF * 8);
  }
  W->total_bytes = (int64_t)W->counter_bytes + kbytes + fbytes;
  W->counters = nullptr;
  W->krec = nullptr;
  W->frec = nullptr;
  if (work) {
    if (reinterpret_cast<uintptr_t>(work) & 255) return PSX_ERR_ARG;
    char* w = static_cast<char*>(work);
    W->counters = reinterpret_cast<int32_t*>(w);
    W->krec = w + W->counter_bytes;
    W->frec = reinterpret_cast<double*>(w + W->counter_bytes + kbytes);
  }
  return PSX_OK;
}

// Queue arguments of one launch: the K queue (sweeps with pair gathers) or the f / K.v
// queue, on the workspace layout W.
inline QueueArgs queue_args(const psx_plan_t* P, const WorkLayout& W, bool queue_k) {
  QueueArgs Q;
  Q.tasks = reinterpret_cast<const int4*>(queue_k ? P->tasks_k : P->tasks_f);
  Q.n_tasks = (int32_t)(queue_k ? P->n_tasks_k : P->n_tasks_f);
  Q.n_granules = P->n_granules;
  Q.btiles = queue_k ? P->btiles_k : P->btiles_f;
  Q.counters = W.counters;
  Q.granule_log2 = W.granule_log2;
  Q.tile = P->tile;
  Q.span_g = W.span_g;
  Q.ring_g = W.ring_g;
  Q.n_elements = P->n_elements;
  Q.max_spins = P->wait_spins > 0 ? P->wait_spins : kDefaultWaitSpins;
  return Q;
}

}  // namespace psx
