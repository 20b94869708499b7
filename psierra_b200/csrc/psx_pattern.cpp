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
