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
