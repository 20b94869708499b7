// Host-side sparsity pattern and node graph (built once per mesh).
//
// The reference builds COO triplets for every element (utility/indexing.py:35-59,
// utility/assembly.py:6-34) and lets scipy's coo_matrix.tocsr() sort and merge them
// on every assembly (utility/assembly.py:75-76).  Here the merged structure is built
// once: for each node the sorted list of distinct neighbour nodes (itself included)
// gives, for DOF row 3i+k, the columns 3j+m (j over the neighbours, m = 0..2) in
// ascending order -- exactly the index arrays scipy produces for those triplets.
#include <algorithm>
#include <cstring>
#include <vector>

#include "psierra_b200.h"

namespace {

bool args_ok(const int64_t* conn, int64_t E, int npe, int64_t N) {
  return conn != nullptr && E >= 0 && N > 0 && (npe == 4 || npe == 10) && N < (int64_t)0x7fffffff &&
         E * npe < (int64_t)0x7fffffff;
}

// Node -> element incidences in ascending element order.
void incidences(const int64_t* conn, int64_t E, int npe, int64_t N, std::vector<int32_t>& ptr,
                std::vector<int32_t>& elem, std::vector<int8_t>& local) {
  ptr.assign(N + 1, 0);
  for (int64_t t = 0; t < E * npe; ++t) ptr[conn[t] + 1]++;
  for (int64_t i = 0; i < N; ++i) ptr[i + 1] += ptr[i];
  elem.resize(E * npe);
  local.resize(E * npe);
  std::vector<int32_t> cur(ptr.begin(), ptr.end() - 1);
  for (int64_t e = 0; e < E; ++e)
    for (int a = 0; a < npe; ++a) {
      int64_t n = conn[e * npe + a];
      int32_t s = cur[n]++;
      elem[s] = (int32_t)e;
      local[s] = (int8_t)a;
    }
}

// Sorted distinct neighbours of node i (incl. i) into `out`.
void neighbours(const int64_t* conn, int npe, const std::vector<int32_t>& ptr,
                const std::vector<int32_t>& elem, int64_t i, std::vector<int32_t>& out) {
  out.clear();
  for (int32_t s = ptr[i]; s < ptr[i + 1]; ++s) {
    const int64_t* c = conn + (int64_t)elem[s] * npe;
    for (int b = 0; b < npe; ++b) out.push_back((int32_t)c[b]);
  }
  std::sort(out.begin(), out.end());
  out.erase(std::unique(out.begin(), out.end()), out.end());
}

bool conn_in_range(const int64_t* conn, int64_t E, int npe, int64_t N) {
  for (int64_t t = 0; t < E * npe; ++t)
    if (conn[t] < 0 || conn[t] >= N) return false;
  return true;
}

}  // namespace

extern "C" int psx_graph_count(const int64_t* conn, int64_t E, int npe, int64_t N, int32_t* nbr_ptr,
                               int32_t* inc_ptr) {
  if (!args_ok(conn, E, npe, N) || !nbr_ptr || !inc_ptr) return PSX_ERR_ARG;
  if (!conn_in_range(conn, E, npe, N)) return PSX_ERR_ARG;
  std::vector<int32_t> ptr, elem;
  std::vector<int8_t> local;
  incidences(conn, E, npe, N, ptr, elem, local);
  std::vector<int32_t> nb;
  int64_t total = 0;
  nbr_ptr[0] = 0;
  for (int64_t i = 0; i < N; ++i) {
    neighbours(conn, npe, ptr, elem, i, nb);
    total += (int64_t)nb.size();
    if (9 * total > (int64_t)0x7fffffff) return PSX_ERR_LIMIT;
    nbr_ptr[i + 1] = (int32_t)total;
  }
  std::memcpy(inc_ptr, ptr.data(), sizeof(int32_t) * (N + 1));
  return PSX_OK;
}

extern "C" int psx_graph_fill(const int64_t* conn, int64_t E, int npe, int64_t N, const int32_t* nbr_ptr,
                              const int32_t* inc_ptr, int32_t* nbr, int32_t* inc_elem, uint32_t* inc_code) {
  if (!args_ok(conn, E, npe, N) || !nbr_ptr || !inc_ptr || !nbr || !inc_elem || !inc_code) return PSX_ERR_ARG;
  if (!conn_in_range(conn, E, npe, N)) return PSX_ERR_ARG;
  std::vector<int32_t> ptr, elem;
  std::vector<int8_t> local;
  incidences(conn, E, npe, N, ptr, elem, local);
  std::vector<int32_t> nb;
  for (int64_t i = 0; i < N; ++i) {
    neighbours(conn, npe, ptr, elem, i, nb);
    if ((int32_t)nb.size() != nbr_ptr[i + 1] - nbr_ptr[i] || ptr[i] != inc_ptr[i]) return PSX_ERR_ARG;
    std::copy(nb.begin(), nb.end(), nbr + nbr_ptr[i]);
    for (int32_t s = ptr[i]; s < ptr[i + 1]; ++s) {
      inc_elem[s] = elem[s];
      uint32_t code = (uint32_t)local[s] & 15u;
      if (npe == 4) {
        code &= 3u;
        const int64_t* c = conn + (int64_t)elem[s] * 4;
        for (int b = 0; b < 4; ++b) {
          int32_t r = (int32_t)(std::lower_bound(nb.begin(), nb.end(), (int32_t)c[b]) - nb.begin());
          if (r >= 128) return PSX_ERR_LIMIT;
          code |= (uint32_t)r << (2 + 7 * b);
        }
      }
      inc_code[s] = code;
    }
  }
  return PSX_OK;
}

extern "C" int psx_csr_pattern(int64_t N, const int32_t* nbr_ptr, const int32_t* nbr, int32_t* indptr,
                               int32_t* indices) {
  if (N <= 0 || !nbr_ptr || !nbr || !indptr || !indices) return PSX_ERR_ARG;
  if (9 * (int64_t)nbr_ptr[N] > (int64_t)0x7fffffff) return PSX_ERR_LIMIT;
  for (int64_t i = 0; i < N; ++i) {
    int32_t b0 = nbr_ptr[i], deg = nbr_ptr[i + 1] - b0;
    for (int k = 0; k < 3; ++k) {
      int32_t start = 9 * b0 + 3 * deg * k;
      indptr[3 * i + k] = start;
      for (int32_t r = 0; r < deg; ++r)
        for (int m = 0; m < 3; ++m) indices[start + 3 * r + m] = 3 * nbr[b0 + r] + m;
    }
  }
  indptr[3 * N] = 9 * nbr_ptr[N];
  return PSX_OK;
}

extern "C" int psx_block_lists(const int64_t* conn, int64_t E, int npe, int64_t N, const int32_t* nbr_ptr,
                               const int32_t* nbr, int32_t* blk_ptr, int32_t* blk_src) {
  if (!args_ok(conn, E, npe, N) || !nbr_ptr || !nbr || !blk_ptr || !blk_src) return PSX_ERR_ARG;
  if (E * npe * npe > (int64_t)0x7fffffff) return PSX_ERR_LIMIT;
  const int64_t nent = nbr_ptr[N];
  std::vector<int32_t> ptr, elem;
  std::vector<int8_t> local;
  incidences(conn, E, npe, N, ptr, elem, local);
  // count per neighbour entry
  std::vector<int32_t> cnt(nent + 1, 0);
  std::vector<int32_t> rank((size_t)npe);
  auto ranks_of = [&](int64_t i, int32_t e) {
    const int32_t* b0 = nbr + nbr_ptr[i];
    const int32_t* b1 = nbr + nbr_ptr[i + 1];
    const int64_t* c = conn + (int64_t)e * npe;
    for (int b = 0; b < npe; ++b) rank[b] = (int32_t)(std::lower_bound(b0, b1, (int32_t)c[b]) - b0);
  };
  for (int64_t i = 0; i < N; ++i)
    for (int32_t s = ptr[i]; s < ptr[i + 1]; ++s) {
      ranks_of(i, elem[s]);
      for (int b = 0; b < npe; ++b) cnt[nbr_ptr[i] + rank[b] + 1]++;
    }
  for (int64_t q = 0; q < nent; ++q) cnt[q + 1] += cnt[q];
  std::memcpy(blk_ptr, cnt.data(), sizeof(int32_t) * (nent + 1));
  std::vector<int32_t> cur(cnt.begin(), cnt.end() - 1);
  for (int64_t i = 0; i < N; ++i)
    for (int32_t s = ptr[i]; s < ptr[i + 1]; ++s) {
      int32_t e = elem[s];
      int a = local[s];
      ranks_of(i, e);
      for (int b = 0; b < npe; ++b) blk_src[cur[nbr_ptr[i] + rank[b]]++] = (e * npe + a) * npe + b;
    }
  return PSX_OK;
}

// ---------------------------------------------------------------------------
// Gather plan for the element-record / owner-gather assembly.
//
// Items: every node pair (i < j) of the node graph ("pair", off-diagonal block K_ij and
// its transpose K_ji) and every node ("node", diagonal block K_ii and f_i).  Each item
// lists its contributing element slots in ascending element order; items are sorted by
// the granule of their "ready" element (the largest contributing element id) and keep
// their (i, j) order inside a granule, so that the items completed by granules [0, g)
// form a prefix and can be gathered right after those elements have been evaluated.
namespace {

inline int local_pair_index(int a, int b, int npe) {  // a < b
  return a * npe - a * (a + 1) / 2 + (b - a - 1);
}

struct Item {
  int32_t ready;
  int32_t order;  // tie break: original item index
};

}  // namespace

extern "C" int psx_plan_count(const int64_t* conn, int64_t E, int npe, int64_t N, const int32_t* nbr_ptr,
                              int64_t* n_pairs, int64_t* n_pair_src) {
  if (!args_ok(conn, E, npe, N) || !nbr_ptr || !n_pairs || !n_pair_src) return PSX_ERR_ARG;
  if (E > ((int64_t)1 << 25)) return PSX_ERR_LIMIT;  // slot encoding e * 64 + slot must fit int32
  *n_pairs = ((int64_t)nbr_ptr[N] - N) / 2;
  *n_pair_src = E * (int64_t)(npe * (npe - 1) / 2);
  return PSX_OK;
}

extern "C" int psx_plan_fill(const int64_t* conn, int64_t E, int npe, int64_t N, const int32_t* nbr_ptr,
                             const int32_t* nbr, int64_t granule, int32_t* pair_info, int32_t* pair_ptr,
                             int32_t* pair_src, int32_t* pair_gptr, int32_t* node_info, int32_t* node_ptr,
                             int32_t* node_src, int32_t* node_gptr, int64_t* max_span) {
  if (!args_ok(conn, E, npe, N) || !nbr_ptr || !nbr || granule <= 0 || !pair_info || !pair_ptr || !pair_src ||
      !pair_gptr || !node_info || !node_ptr || !node_src || !node_gptr || !max_span)
    return PSX_ERR_ARG;
  if (E > ((int64_t)1 << 25)) return PSX_ERR_LIMIT;
  std::vector<int32_t> ptr, elem;
  std::vector<int8_t> local;
  incidences(conn, E, npe, N, ptr, elem, local);
  const int64_t n_pairs = ((int64_t)nbr_ptr[N] - N) / 2;
  const int64_t n_gran = (E + granule - 1) / granule;

  // ---- pairs in (i, j) order: contributions = inc(i) intersect inc(j)
  std::vector<int32_t> p_ptr(n_pairs + 1, 0), p_src;
  std::vector<int32_t> p_info(4 * n_pairs);
  std::vector<Item> p_item(n_pairs);
  std::vector<int32_t> p_min(n_pairs);
  p_src.reserve((size_t)E * (npe * (npe - 1) / 2));
  int64_t p = 0;
  for (int64_t i = 0; i < N; ++i) {
    const int32_t b0 = nbr_ptr[i], deg = nbr_ptr[i + 1] - b0;
    for (int32_t r = 0; r < deg; ++r) {
      const int64_t j = nbr[b0 + r];
      if (j <= i) continue;
      const int32_t* ej = nbr + nbr_ptr[j];
      const int32_t degj = nbr_ptr[j + 1] - nbr_ptr[j];
      const int32_t rji = (int32_t)(std::lower_bound(ej, ej + degj, (int32_t)i) - ej);
      p_info[4 * p + 0] = 9 * b0 + 3 * r;
      p_info[4 * p + 1] = 3 * deg;
      p_info[4 * p + 2] = 9 * nbr_ptr[j] + 3 * rji;
      p_info[4 * p + 3] = 3 * degj;
      int32_t si = ptr[i], sj = ptr[j], emax = -1, emin = 0x7fffffff;
      while (si < ptr[i + 1] && sj < ptr[j + 1]) {
        if (elem[si] < elem[sj]) {
          ++si;
        } else if (elem[si] > elem[sj]) {
          ++sj;
        } else {
          const int a = local[si], b = local[sj];
          const int slot = local_pair_index(std::min(a, b), std::max(a, b), npe);
          p_src.push_back(elem[si] * 64 + slot);
          emax = std::max(emax, elem[si]);
          emin = std::min(emin, elem[si]);
          ++si;
          ++sj;
        }
      }
      if (emax < 0) return PSX_ERR_ARG;  // a graph edge must come from some element
      p_ptr[p + 1] = (int32_t)p_src.size();
      p_item[p] = {emax, (int32_t)p};
      p_min[p] = emin;
      ++p;
    }
  }
  if (p != n_pairs) return PSX_ERR_ARG;

  // ---- nodes: contributions = inc(i)
  std::vector<Item> n_item(N);
  int64_t span = 0;
  for (int64_t i = 0; i < N; ++i) {
    if (ptr[i + 1] == ptr[i]) {
      n_item[i] = {-1, (int32_t)i};  // isolated node: ready before everything
      continue;
    }
    const int32_t emin = elem[ptr[i]], emax = elem[ptr[i + 1] - 1];
    n_item[i] = {emax, (int32_t)i};
    span = std::max<int64_t>(span, emax - emin);
  }
  for (int64_t q = 0; q < n_pairs; ++q) span = std::max<int64_t>(span, p_item[q].ready - p_min[q]);
  *max_span = span;

  auto by_ready = [](const Item& x, const Item& y) {
    return x.ready < y.ready || (x.ready == y.ready && x.order < y.order);
  };
  // Within a granule, items keep (i, j) order (their original order), so that lanes of a
  // gather tile write neighbouring blocks of the same CSR rows.
  auto by_granule = [granule](const Item& x, const Item& y) {
    const int64_t gx = x.ready < 0 ? -1 : x.ready / granule, gy = y.ready < 0 ? -1 : y.ready / granule;
    return gx < gy || (gx == gy && x.order < y.order);
  };
  std::sort(p_item.begin(), p_item.end(), by_granule);
  std::sort(n_item.begin(), n_item.end(), by_granule);
  (void)by_ready;

  // ---- emit pairs in ready order
  int32_t out = 0;
  pair_ptr[0] = 0;
  for (int64_t k = 0; k < n_pairs; ++k) {
    const int32_t q = p_item[k].order;
    std::memcpy(pair_info + 4 * k, p_info.data() + 4 * q, 4 * sizeof(int32_t));
    for (int32_t s = p_ptr[q]; s < p_ptr[q + 1]; ++s) pair_src[out++] = p_src[s];
    pair_ptr[k + 1] = out;
  }
  // granule ranges: items whose ready element lies in granule g
  {
    int64_t k = 0;
    for (int64_t g = 0; g <= n_gran; ++g) {
      const int64_t limit = std::min<int64_t>(E, g * granule);  // ready < limit
      while (k < n_pairs && p_item[k].ready < limit) ++k;
      pair_gptr[g] = (int32_t)k;
    }
    pair_gptr[n_gran] = (int32_t)n_pairs;
  }
  // ---- emit nodes in ready order
  out = 0;
  node_ptr[0] = 0;
  for (int64_t k = 0; k < N; ++k) {
    const int32_t i = n_item[k].order;
    const int32_t b0 = nbr_ptr[i], deg = nbr_ptr[i + 1] - b0;
    const int32_t rii = (int32_t)(std::lower_bound(nbr + b0, nbr + b0 + deg, i) - (nbr + b0));
    node_info[4 * k + 0] = 9 * b0 + 3 * rii;
    node_info[4 * k + 1] = 3 * deg;
    node_info[4 * k + 2] = i;
    node_info[4 * k + 3] = 0;
    for (int32_t s = ptr[i]; s < ptr[i + 1]; ++s) node_src[out++] = elem[s] * 16 + local[s];
    node_ptr[k + 1] = out;
  }
  {
    int64_t k = 0;
    for (int64_t g = 0; g <= n_gran; ++g) {
      const int64_t limit = std::min<int64_t>(E, g * granule);
      while (k < N && n_item[k].ready < limit) ++k;
      node_gptr[g] = (int32_t)k;
    }
    node_gptr[n_gran] = (int32_t)N;
  }
  return PSX_OK;
}

// ---------------------------------------------------------------------------
// Tile plan (Tet4): the element tile of one warp (T consecutive elements) sums the
// blocks its elements share before anything leaves the SM.  Per tile, the distinct
// node pairs (and nodes) get local indices by descending contribution count, ties in
// order of first occurrence; for each
// local pair the tile lists its contributions (element-in-tile * 8 + slot) in element
// order.  Everything one tile needs is one contiguous block (psx_tile_meta_stride
// bytes, a multiple of 16) so that a warp copies it to shared memory in one go:
//   [0] np  [1] nn  [2..3] 0
//   node offsets  (nn + 1 bytes, in a 4-byte-rounded field of 4T + 1)
//   node codes    (4T bytes, element-in-tile * 4 + local node)
//   pair offsets  (np + 1 bytes, in a 4-byte-rounded field of 6T + 1)
//   pair codes    (6T bytes, by local pair, element order within a pair)
// The node lists come first: the sweeps without a tangent copy only that prefix.
// The gather lists then name (tile, local index) records instead of element slots, and
// consecutive contributions of one tile collapse into one.
namespace {
inline int64_t up4(int64_t b) { return (b + 3) / 4 * 4; }
struct TileMeta {
  int64_t off_p, off_n, src_p, src_n, stride;
  explicit TileMeta(int64_t T) {
    off_n = 4;
    src_n = off_n + up4(4 * T + 1);
    off_p = src_n + 4 * T;
    src_p = off_p + up4(6 * T + 1);
    stride = (src_p + 6 * T + 15) / 16 * 16;
  }
};
}  // namespace

extern "C" int64_t psx_tile_meta_stride(int32_t T) { return T > 0 ? TileMeta(T).stride : 0; }

extern "C" int psx_tile_plan_fill(const int64_t* conn, int64_t E, int npe, int32_t T, const int32_t* pair_ptr,
                                  const int32_t* pair_src, int64_t n_pairs, const int32_t* node_ptr,
                                  const int32_t* node_src, int64_t N, uint8_t* meta, int32_t* pair_ptr_t,
                                  int32_t* pair_src_t, int32_t* node_ptr_t, int32_t* node_src_t, int32_t* caps) {
  if (!args_ok(conn, E, npe, N) || npe != 4 || T <= 0 || T > 32 || (T & (T - 1)) || !pair_ptr || !pair_src ||
      !node_ptr || !node_src || !meta || !pair_ptr_t || !pair_src_t || !node_ptr_t || !node_src_t || !caps ||
      n_pairs < 0)
    return PSX_ERR_ARG;
  constexpr int kP = 6;  // local pairs of a Tet4
  const int64_t n_tiles = (E + T - 1) / T;
  if (n_tiles >= ((int64_t)1 << 23)) return PSX_ERR_LIMIT;  // codes t * 256 + lp must fit int32
  const TileMeta M(T);
  static const int pa[kP] = {0, 0, 0, 1, 1, 2}, pb[kP] = {1, 2, 3, 2, 3, 3};  // local_pair_index order
  std::vector<uint8_t> slot_lp((size_t)E * kP), node_ln((size_t)E * 4);
  std::vector<std::pair<int64_t, int32_t>> keys;
  keys.reserve(kP * T);
  std::vector<std::pair<int32_t, int32_t>> first;
  int32_t cap_p = 0, cap_n = 0;
  std::memset(meta, 0, (size_t)(n_tiles * M.stride));
  // Group (key, code) entries of one tile: local indices by descending group size, ties
  // in order of first occurrence, each group's codes ascending.  Writes codes to src and offsets to off.
  auto group = [&](uint8_t* src, uint8_t* off, std::vector<uint8_t>& map, int64_t e0, int per,
                   int shift) -> int32_t {
    std::sort(keys.begin(), keys.end());  // by key, then code
    first.clear();                         // (first code, start in keys)
    for (size_t k = 0; k < keys.size(); ++k)
      if (k == 0 || keys[k].first != keys[k - 1].first) first.push_back({keys[k].second, (int32_t)k});
    // local numbering: most contributions first (ties by first occurrence), so that the
    // 32 items a warp sums in one round have similar loop lengths
    auto count = [&](const std::pair<int32_t, int32_t>& f) {
      size_t k = (size_t)f.second;
      while (k < keys.size() && keys[k].first == keys[(size_t)f.second].first) ++k;
      return (int32_t)(k - (size_t)f.second);
    };
    std::sort(first.begin(), first.end(), [&](const auto& x, const auto& y) {
      const int32_t cx = count(x), cy = count(y);
      return cx != cy ? cx > cy : x.first < y.first;
    });
    int32_t pos = 0, local = 0;
    for (const auto& f : first) {
      off[local] = (uint8_t)pos;
      for (size_t k = f.second; k < keys.size() && keys[k].first == keys[f.second].first; ++k) {
        const int32_t code = keys[k].second;
        src[pos++] = (uint8_t)code;
        map[(size_t)(e0 + (code >> shift)) * per + (code & ((1 << shift) - 1))] = (uint8_t)local;
      }
      ++local;
    }
    off[local] = (uint8_t)pos;
    return local;
  };
  for (int64_t t = 0; t < n_tiles; ++t) {
    const int64_t e0 = t * T, e1 = std::min<int64_t>(E, e0 + T);
    uint8_t* m = meta + t * M.stride;
    keys.clear();
    for (int64_t e = e0; e < e1; ++e)
      for (int s = 0; s < kP; ++s) {
        const int64_t i = conn[e * 4 + pa[s]], j = conn[e * 4 + pb[s]];
        keys.push_back({std::min(i, j) * N + std::max(i, j), (int32_t)((e - e0) * 8 + s)});
      }
    const int32_t np = group(m + M.src_p, m + M.off_p, slot_lp, e0, kP, 3);
    keys.clear();
    for (int64_t e = e0; e < e1; ++e)
      for (int a = 0; a < 4; ++a) keys.push_back({conn[e * 4 + a], (int32_t)((e - e0) * 4 + a)});
    const int32_t nn = group(m + M.src_n, m + M.off_n, node_ln, e0, 4, 2);
    m[0] = (uint8_t)np;
    m[1] = (uint8_t)nn;
    cap_p = std::max(cap_p, np);
    cap_n = std::max(cap_n, nn);
  }
  int32_t lg = 0;
  while ((1 << lg) < T) ++lg;
  // gather lists: element codes -> (tile, local) codes, consecutive duplicates merged
  int64_t out = 0;
  pair_ptr_t[0] = 0;
  for (int64_t k = 0; k < n_pairs; ++k) {
    int64_t last = -1;
    for (int32_t q = pair_ptr[k]; q < pair_ptr[k + 1]; ++q) {
      const int64_t e = pair_src[q] >> 6, slot = pair_src[q] & 63;
      const int64_t c = (e >> lg) * 256 + slot_lp[(size_t)e * kP + slot];
      if (c != last) pair_src_t[out++] = (int32_t)c;
      last = c;
    }
    pair_ptr_t[k + 1] = (int32_t)out;
  }
  out = 0;
  node_ptr_t[0] = 0;
  for (int64_t k = 0; k < N; ++k) {
    int64_t last = -1;
    for (int32_t q = node_ptr[k]; q < node_ptr[k + 1]; ++q) {
      const int64_t e = node_src[q] >> 4, a = node_src[q] & 15;
      const int64_t c = (e >> lg) * 128 + node_ln[(size_t)e * 4 + a];
      if (c != last) node_src_t[out++] = (int32_t)c;
      last = c;
    }
    node_ptr_t[k + 1] = (int32_t)out;
  }
  caps[0] = cap_p;
  caps[1] = cap_n;
  return PSX_OK;
}

// ---------------------------------------------------------------------------
// F-bar plan (Tet4Fbar, element/tet4_fbar.py:53-118, 420-459).  The nodal volumetric
// blocks kappa v0_a g_a g_a^T couple every two nodes of node a's element patch, so the
// tangent lives on the two-ring graph: b ~ c when some node a neighbours both.  For
// each two-ring block (b, c) the plan lists the nodes a it sums over (ascending, the
// order of the reference's COO -> CSR accumulation) with the one-ring entries of g_a[b]
// and g_a[c]; the one-ring gather items get their positions in the two-ring CSR.
namespace {
inline int32_t rank_in(const int32_t* list, int32_t n, int32_t v) {
  return (int32_t)(std::lower_bound(list, list + n, v) - list);
}
}  // namespace

extern "C" int psx_fbar_plan_count(int64_t N, const int32_t* nbr_ptr, const int32_t* nbr, int64_t* n_nbr2,
                                   int64_t* n_vol) {
  if (N <= 0 || !nbr_ptr || !nbr || !n_nbr2 || !n_vol) return PSX_ERR_ARG;
  std::vector<int32_t> mark(N, -1);
  int64_t tot = 0, vol = 0;
  for (int64_t b = 0; b < N; ++b) {
    for (int32_t x = nbr_ptr[b]; x < nbr_ptr[b + 1]; ++x) {
      const int32_t a = nbr[x];
      for (int32_t y = nbr_ptr[a]; y < nbr_ptr[a + 1]; ++y)
        if (mark[nbr[y]] != (int32_t)b) {
          mark[nbr[y]] = (int32_t)b;
          ++tot;
        }
    }
  }
  for (int64_t a = 0; a < N; ++a) {
    const int64_t d = nbr_ptr[a + 1] - nbr_ptr[a];
    vol += d * d;
  }
  if (9 * tot >= ((int64_t)1 << 31) || 3 * vol >= ((int64_t)1 << 31)) return PSX_ERR_LIMIT;
  *n_nbr2 = tot;
  *n_vol = vol;
  return PSX_OK;
}

extern "C" int psx_fbar_plan_fill(int64_t N, const int32_t* nbr_ptr, const int32_t* nbr, int64_t n_pairs,
                                  const int32_t* pair_info, const int32_t* node_info, int32_t* nbr2_ptr,
                                  int32_t* nbr2, int32_t* pair_info2, int32_t* node_info2, int32_t* vol_ptr,
                                  int32_t* vol_src) {
  if (N <= 0 || !nbr_ptr || !nbr || n_pairs < 0 || !pair_info || !node_info || !nbr2_ptr || !nbr2 ||
      !pair_info2 || !node_info2 || !vol_ptr || !vol_src)
    return PSX_ERR_ARG;
  // two-ring neighbour lists (sorted, self included)
  std::vector<int32_t> tmp;
  nbr2_ptr[0] = 0;
  for (int64_t b = 0; b < N; ++b) {
    tmp.clear();
    for (int32_t x = nbr_ptr[b]; x < nbr_ptr[b + 1]; ++x) {
      const int32_t a = nbr[x];
      tmp.insert(tmp.end(), nbr + nbr_ptr[a], nbr + nbr_ptr[a + 1]);
    }
    std::sort(tmp.begin(), tmp.end());
    tmp.erase(std::unique(tmp.begin(), tmp.end()), tmp.end());
    std::copy(tmp.begin(), tmp.end(), nbr2 + nbr2_ptr[b]);
    nbr2_ptr[b + 1] = nbr2_ptr[b] + (int32_t)tmp.size();
  }
  auto rank2 = [&](int32_t i, int32_t j) { return rank_in(nbr2 + nbr2_ptr[i], nbr2_ptr[i + 1] - nbr2_ptr[i], j); };
  // one-ring gather positions -> two-ring CSR positions
  for (int64_t k = 0; k < n_pairs; ++k) {
    const int32_t pos = pair_info[4 * k];
    // row node i: 9 nbr_ptr[i] <= pos < 9 nbr_ptr[i + 1]
    const int32_t i = (int32_t)(std::upper_bound(nbr_ptr, nbr_ptr + N + 1, pos / 9) - nbr_ptr) - 1;
    const int32_t r = (pos - 9 * nbr_ptr[i]) / 3;
    const int32_t j = nbr[nbr_ptr[i] + r];
    const int32_t deg2i = nbr2_ptr[i + 1] - nbr2_ptr[i], deg2j = nbr2_ptr[j + 1] - nbr2_ptr[j];
    pair_info2[4 * k + 0] = 9 * nbr2_ptr[i] + 3 * rank2(i, j);
    pair_info2[4 * k + 1] = 3 * deg2i;
    pair_info2[4 * k + 2] = 9 * nbr2_ptr[j] + 3 * rank2(j, i);
    pair_info2[4 * k + 3] = 3 * deg2j;
  }
  for (int64_t k = 0; k < N; ++k) {
    const int32_t i = node_info[4 * k + 2];
    const int32_t deg2i = nbr2_ptr[i + 1] - nbr2_ptr[i];
    node_info2[4 * k + 0] = 9 * nbr2_ptr[i] + 3 * rank2(i, i);
    node_info2[4 * k + 1] = node_info[4 * k + 1] > 0 ? 3 * deg2i : 0;
    node_info2[4 * k + 2] = i;
    node_info2[4 * k + 3] = 0;
  }
  // volumetric lists: for block (b, c), the common one-ring neighbours a of b and c
  int64_t out = 0;
  vol_ptr[0] = 0;
  for (int64_t b = 0; b < N; ++b) {
    const int32_t* nb = nbr + nbr_ptr[b];
    const int32_t db = nbr_ptr[b + 1] - nbr_ptr[b];
    for (int32_t t = nbr2_ptr[b]; t < nbr2_ptr[b + 1]; ++t) {
      const int32_t c = nbr2[t];
      const int32_t* nc = nbr + nbr_ptr[c];
      const int32_t dc = nbr_ptr[c + 1] - nbr_ptr[c];
      int32_t x = 0, y = 0;
      while (x < db && y < dc) {
        if (nb[x] < nc[y]) {
          ++x;
        } else if (nb[x] > nc[y]) {
          ++y;
        } else {
          const int32_t a = nb[x];
          const int32_t* na = nbr + nbr_ptr[a];
          const int32_t da = nbr_ptr[a + 1] - nbr_ptr[a];
          vol_src[3 * out + 0] = a;
          vol_src[3 * out + 1] = nbr_ptr[a] + rank_in(na, da, (int32_t)b);
          vol_src[3 * out + 2] = nbr_ptr[a] + rank_in(na, da, c);
          ++out;
          ++x;
          ++y;
        }
      }
      vol_ptr[t + 1] = (int32_t)out;
    }
  }
  return PSX_OK;
}

// ---------------------------------------------------------------------------
// Task queue of the persistent assembly kernel: for each granule g, the element
// tiles of g followed by the gather tiles made ready by granule g-1-lag (pairs, then
// nodes); the gather tiles of the last granules close the queue.  The lag keeps gather
// tiles from being claimed while the element tiles they read are still running.  Task = int4
// {kind, granule, begin, end}: kind 0 = element tile [begin, end), 1 = pair items,
// 2 = node items.  `with_pairs` = 0 builds the f-only queue (no pair tiles).
extern "C" int psx_task_count(const psx_plan_t* P, int with_pairs, int32_t tile, int32_t tile_items, int32_t lag,
                              int64_t* n_tasks) {
  if (!P || !P->pair_gptr || !P->node_gptr || tile <= 0 || tile_items <= 0 || P->granule % tile || lag < 0 ||
      !n_tasks)
    return PSX_ERR_ARG;
  int64_t n = 0;
  const int64_t G = P->n_granules;
  for (int64_t g = 0; g <= G + lag; ++g) {
    if (g < G) {
      const int64_t e0 = g * P->granule, e1 = std::min<int64_t>(P->n_elements, e0 + P->granule);
      n += (e1 - e0 + tile - 1) / tile;
    }
    if (g >= 1 + lag && g - 1 - lag < G) {
      const int64_t r = g - 1 - lag;
      if (with_pairs) n += (P->pair_gptr[r + 1] - P->pair_gptr[r] + tile_items - 1) / tile_items;
      const int64_t n0 = r == 0 ? 0 : P->node_gptr[r];
      n += (P->node_gptr[r + 1] - n0 + tile_items - 1) / tile_items;
    }
  }
  *n_tasks = n;
  return PSX_OK;
}

extern "C" int psx_task_fill(const psx_plan_t* P, int with_pairs, int32_t tile, int32_t tile_items, int32_t lag,
                             int32_t* tasks, int32_t* b_tiles_per_granule) {
  if (!P || !P->pair_gptr || !P->node_gptr || tile <= 0 || tile_items <= 0 || P->granule % tile || lag < 0 ||
      !tasks || !b_tiles_per_granule)
    return PSX_ERR_ARG;
  const int64_t G = P->n_granules;
  int64_t k = 0;
  auto push = [&](int32_t kind, int64_t g, int64_t b, int64_t e) {
    tasks[4 * k + 0] = kind;
    tasks[4 * k + 1] = (int32_t)g;
    tasks[4 * k + 2] = (int32_t)b;
    tasks[4 * k + 3] = (int32_t)e;
    ++k;
  };
  for (int64_t g = 0; g <= G + lag; ++g) {
    if (g < G) {
      const int64_t e0 = g * P->granule, e1 = std::min<int64_t>(P->n_elements, e0 + P->granule);
      for (int64_t b = e0; b < e1; b += tile) push(0, g, b, std::min<int64_t>(e1, b + tile));
    }
    if (g >= 1 + lag && g - 1 - lag < G) {
      const int64_t r = g - 1 - lag;
      int32_t nb = 0;
      if (with_pairs)
        for (int64_t b = P->pair_gptr[r]; b < P->pair_gptr[r + 1]; b += tile_items, ++nb)
          push(1, r, b, std::min<int64_t>(P->pair_gptr[r + 1], b + tile_items));
      const int64_t n0 = r == 0 ? 0 : P->node_gptr[r];
      for (int64_t b = n0; b < P->node_gptr[r + 1]; b += tile_items, ++nb)
        push(2, r, b, std::min<int64_t>(P->node_gptr[r + 1], b + tile_items));
      b_tiles_per_granule[r] = nb;
    }
  }
  return PSX_OK;
}
