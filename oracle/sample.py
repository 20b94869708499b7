"""Rows of the assembled f_int and K_T for a sample of nodes, from the reference algorithm.

Test infrastructure only (the checker of large configurations, where the complete
COO->CSR assembly of every element would not fit a test's time or memory).

The global f entry and K row of DOF ``3 n + c`` are sums over the elements that contain
node ``n`` and nothing else (psierra ``utility/assembly.py:37-108``: every element
contributes only to the rows of its own DOFs).  So evaluating exactly the elements
incident to the sampled nodes with the reference element
(``element/tet4_total_lagrangian.py:77-139`` or ``element/tet10_total_lagrangian.py:63-136``,
batched in ``oracle.vectorized``) and assembling them with the reference's COO->CSR
summation gives those rows completely; the rows of other nodes are dropped.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as spsp

from oracle import vectorized
from oracle.assembly import coo_indices, element_dofs


def sample_nodes(n_nodes: int, count: int, seed: int) -> np.ndarray:
    """``count`` distinct node ids, sorted, from a seeded generator."""
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(n_nodes, size=min(count, n_nodes), replace=False))


def sampled_rows(nodes, elements, u, mu, kappa, sample, chunk: int = 50000):
    """``(dofs, K_rows, f_rows)`` for the sampled nodes.

    ``dofs`` are the sampled nodes' DOFs ascending (3 per node); ``K_rows`` is a CSR of
    shape ``(len(dofs), 3 N)`` whose row i is the global row ``dofs[i]``; ``f_rows`` the
    f_int entries of those DOFs.  ``mu``/``kappa`` are scalars or per-element arrays.
    """
    el = np.asarray(elements, dtype=np.int64)
    E, npe = el.shape
    n_dofs = 3 * nodes.shape[0]
    in_sample = np.zeros(nodes.shape[0], dtype=bool)
    in_sample[np.asarray(sample)] = True
    touched = np.flatnonzero(in_sample[el].any(axis=1))  # ascending: element order kept
    mu_e = np.broadcast_to(np.asarray(mu, dtype=np.float64), (E,))
    ka_e = np.broadcast_to(np.asarray(kappa, dtype=np.float64), (E,))
    dofs = np.sort(np.concatenate([3 * np.asarray(sample) + c for c in range(3)]))
    row_of = -np.ones(n_dofs, dtype=np.int64)
    row_of[dofs] = np.arange(dofs.size)
    rows, cols, vals = [], [], []
    f = np.zeros(dofs.size)
    for a in range(0, touched.size, chunk):
        idx = touched[a:a + chunk]
        k, fe = vectorized.element_force_and_tangent(nodes, el[idx], u, mu_e[idx], ka_e[idx])
        ed = element_dofs(el[idx])
        r, c = coo_indices(ed)
        keep = row_of[r] >= 0
        rows.append(row_of[r[keep]])
        cols.append(c[keep])
        vals.append(k.reshape(-1)[keep])
        fk = row_of[ed.reshape(-1)]
        sel = fk >= 0
        np.add.at(f, fk[sel], fe.reshape(-1)[sel])  # element order, like assemble_vector
    K = spsp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                        shape=(dofs.size, n_dofs)).tocsr()
    return dofs, K, f


def gpu_rows(indptr, indices, values, dofs):
    """CSR of the rows ``dofs`` of a full matrix given by its CSR arrays (host numpy)."""
    n = indptr.size - 1
    A = spsp.csr_matrix((np.asarray(values, dtype=np.float64), indices, indptr), shape=(n, n))
    return A[dofs]


def compare_rows(K_gpu_rows, K_ref_rows) -> tuple[bool, float]:
    """(same pattern, max |K - K_ref| / max |K_ref|) of two row sets with sorted indices."""
    a = K_gpu_rows.tocsr()
    b = K_ref_rows.tocsr()
    a.sort_indices()
    b.sort_indices()
    same = np.array_equal(a.indptr, b.indptr) and np.array_equal(a.indices, b.indices)
    if not same:
        return False, float("inf")
    return True, float(np.abs(a.data - b.data).max() / np.abs(b.data).max())
