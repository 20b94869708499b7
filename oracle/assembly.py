"""Global assembly restated from psierra ``utility/indexing.py``, ``utility/assembly.py``
and ``domain/solid.py``.  Test infrastructure only.

Per-element material: the reference ``NeoHookean`` holds one scalar (mu, K)
(``material/neohookean.py:83-84``).  ``mu``/``kappa`` here may be scalars or
per-element arrays; an array restates "one NeoHookean per element", which is
how the per-element parameters of the adjoint path are checked.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as spsp

from oracle import tet4, tet10


def element_dofs(elements: np.ndarray) -> np.ndarray:
    """``indexing.py:35-59``: dof = 3*node + c, row-major per element."""
    el = np.asarray(elements, dtype=np.int64)
    return (el[:, :, None] * 3 + np.arange(3)[None, None, :]).reshape(el.shape[0], -1)


def coo_indices(edofs: np.ndarray):
    """``assembly.py:6-34``: rows/cols broadcast over the (d x d) local grid."""
    n, d = edofs.shape
    rows = np.broadcast_to(edofs[:, :, None], (n, d, d)).reshape(-1)
    cols = np.broadcast_to(edofs[:, None, :], (n, d, d)).reshape(-1)
    return rows, cols


def assemble_sparse(kloc: np.ndarray, rows, cols, n_dofs: int) -> spsp.csr_matrix:
    """``assembly.py:37-76``: ``coo_matrix(...).tocsr()`` (sums duplicates, sorted)."""
    data = np.asarray(kloc, dtype=np.float64).reshape(-1)
    return spsp.coo_matrix((data, (rows, cols)), shape=(n_dofs, n_dofs)).tocsr()


def assemble_vector(floc: np.ndarray, edofs: np.ndarray, n_dofs: int) -> np.ndarray:
    """``assembly.py:79-108``: ``np.add.at`` in element order."""
    g = np.zeros(n_dofs, dtype=np.float64)
    np.add.at(g, edofs.ravel(), floc.ravel())
    return g


def _per_elem(v, n):
    a = np.asarray(v, dtype=np.float64)
    return np.broadcast_to(a, (n,)) if a.ndim == 0 else a


def _element_module(npe: int):
    return tet4 if npe == 4 else tet10


def element_loop(nodes, elements, u_nodes, mu, kappa):
    """Per-element (k, f) exactly as ``solid.py:252-268`` / ``:302-318`` compute them."""
    el = np.asarray(elements, dtype=np.int64)
    E, npe = el.shape
    mod = _element_module(npe)
    mus, ks = _per_elem(mu, E), _per_elem(kappa, E)
    d = 3 * npe
    kl = np.zeros((E, d, d))
    fl = np.zeros((E, d))
    for e in range(E):
        idx = el[e]
        kl[e], fl[e] = mod.force_and_tangent(nodes[idx], u_nodes[idx], mus[e], ks[e])
    return kl, fl


def assemble_internal_forces(nodes, elements, u_nodes, mu, kappa) -> np.ndarray:
    """``SolidDomain.assemble_internal_forces`` (``solid.py:230-274``)."""
    _, fl = element_loop(nodes, elements, u_nodes, mu, kappa)
    ed = element_dofs(elements)
    return assemble_vector(fl, ed, 3 * nodes.shape[0])


def assemble_tangent(nodes, elements, u_nodes, mu, kappa) -> spsp.csr_matrix:
    """``SolidDomain.assemble_tangent_stiffness_matrix`` (``solid.py:280-325``)."""
    kl, _ = element_loop(nodes, elements, u_nodes, mu, kappa)
    ed = element_dofs(elements)
    r, c = coo_indices(ed)
    return assemble_sparse(kl, r, c, 3 * nodes.shape[0])


def assemble_force_and_tangent(nodes, elements, u_nodes, mu, kappa):
    """Both outputs from one element sweep (same values as the two reference sweeps)."""
    kl, fl = element_loop(nodes, elements, u_nodes, mu, kappa)
    ed = element_dofs(elements)
    r, c = coo_indices(ed)
    n = 3 * nodes.shape[0]
    return assemble_vector(fl, ed, n), assemble_sparse(kl, r, c, n)


def assemble_linear_stiffness(nodes, elements, lam, mu) -> spsp.csr_matrix:
    """``SolidDomain.assemble_stiffness_matrix`` (``solid.py:172-207``)."""
    el = np.asarray(elements, dtype=np.int64)
    E, npe = el.shape
    mod = _element_module(npe)
    lams, mus = _per_elem(lam, E), _per_elem(mu, E)
    kl = np.stack([mod.linear_stiffness(nodes[el[e]], lams[e], mus[e]) for e in range(E)])
    ed = element_dofs(el)
    r, c = coo_indices(ed)
    return assemble_sparse(kl, r, c, 3 * nodes.shape[0])


def assemble_mass(nodes, elements, rho) -> spsp.csr_matrix:
    """``SolidDomain.assemble_mass_matrix`` (``solid.py:209-228``) for Tet4."""
    el = np.asarray(elements, dtype=np.int64)
    X = nodes[el[:, :4]]
    vols = np.abs(np.linalg.det(X[:, 1:4] - X[:, 0:1])) / 6.0
    kl = np.stack([tet4.mass_matrix(rho, v) for v in vols])
    ed = element_dofs(el)
    r, c = coo_indices(ed)
    return assemble_sparse(kl, r, c, 3 * nodes.shape[0])
