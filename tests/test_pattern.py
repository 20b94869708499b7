"""Host-side pattern logic and the C ABI surface (CPU only).

* the library loads and exports every entry point declared in ``include/*.h``;
* the CSR index arrays equal scipy's ``coo_matrix(...).tocsr()`` of the reference's
  COO triplets bit for bit (psierra ``utility/assembly.py:6-34, 75-76``);
* the node-centric slot map reproduces scipy's duplicate summation exactly
  (integer-valued element matrices, so any ordering gives the same sums);
* the Tet10 gather lists do the same for the element-centric path.
"""
from __future__ import annotations

import glob
import os
import re

import numpy as np
import pytest
import scipy.sparse as spsp

from conftest import ROOT
from oracle.assembly import coo_indices, element_dofs
from psierra_b200 import _lib, meshgen
from psierra_b200.pattern import MeshPattern


def declared_symbols() -> list[str]:
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        names += re.findall(r"^\s*(?:int|int64_t|size_t|void)\s+(psx_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = declared_symbols()
    assert len(names) >= 7
    for n in names:
        assert hasattr(L, n), f"{n} declared in include/ but not exported"
    assert L.psx_status_bytes() == 32


def _scipy_pattern(elements, n_dofs):
    ed = element_dofs(elements)
    r, c = coo_indices(ed)
    return spsp.coo_matrix((np.ones(r.size), (r, c)), shape=(n_dofs, n_dofs)).tocsr(), r, c


def _random_unstructured(seed=0):
    """Randomly renumbered Kuhn box with shuffled element order (an 'unstructured' mesh)."""
    rng = np.random.default_rng(seed)
    m = meshgen.box_tet4(1.0, 0.7, 0.5, 5, 4, 3)
    perm = rng.permutation(m.n_nodes)
    inv = np.empty_like(perm)
    inv[perm] = np.arange(m.n_nodes)
    els = inv[m.elements][rng.permutation(m.n_elements)]
    return meshgen.TetMesh(m.nodes[perm], els)


MESHES = {
    "cfg1": lambda: meshgen.box_tet4(1.0, 0.1, 0.1, 40, 4, 4),
    "unstructured": _random_unstructured,
    "tet10": lambda: meshgen.tet4_to_tet10(meshgen.box_tet4(1.0, 1.0, 1.0, 3, 2, 2)),
    "single": lambda: meshgen.TetMesh(np.eye(4, 3, k=-1) + 0.0, np.array([[0, 1, 2, 3]])),
}


@pytest.mark.parametrize("name", sorted(MESHES))
def test_csr_pattern_bit_exact(name):
    m = MESHES[name]()
    p = MeshPattern(m.elements, m.n_nodes)
    A, _, _ = _scipy_pattern(m.elements, m.n_dofs)
    assert p.indptr.dtype == A.indptr.dtype == np.int32
    assert np.array_equal(p.indptr, A.indptr)
    assert np.array_equal(p.indices, A.indices)
    assert p.nnz == A.nnz


@pytest.mark.parametrize("name", ["cfg1", "unstructured", "single"])
def test_tet4_slot_map_reproduces_coo_sum(name):
    m = MESHES[name]()
    p = MeshPattern(m.elements, m.n_nodes)
    E = m.n_elements
    rng = np.random.default_rng(1)
    kl = rng.integers(-1000, 1000, size=(E, 12, 12)).astype(np.float64)
    _, r, c = _scipy_pattern(m.elements, m.n_dofs)
    B = spsp.coo_matrix((kl.ravel(), (r, c)), shape=(m.n_dofs,) * 2).tocsr()
    vals = np.zeros(p.nnz)
    for i in range(m.n_nodes):
        deg = p.nbr_ptr[i + 1] - p.nbr_ptr[i]
        base = 9 * p.nbr_ptr[i]
        for s in range(p.inc_ptr[i], p.inc_ptr[i + 1]):
            e, code = p.inc_elem[s], int(p.inc_code[s])
            a = code & 3
            assert m.elements[e, a] == i
            for b in range(4):
                rb = (code >> (2 + 7 * b)) & 127
                blk = kl[e, 3 * a:3 * a + 3, 3 * b:3 * b + 3]
                for k in range(3):
                    vals[base + 3 * deg * k + 3 * rb: base + 3 * deg * k + 3 * rb + 3] += blk[k]
    assert np.array_equal(vals, B.data)


def test_block_lists_reproduce_coo_sum():
    m = MESHES["tet10"]()
    p = MeshPattern(m.elements, m.n_nodes)
    blk_ptr, blk_src = p.block_lists()
    E, npe = m.elements.shape
    rng = np.random.default_rng(2)
    kl = rng.integers(-1000, 1000, size=(E, 3 * npe, 3 * npe)).astype(np.float64)
    _, r, c = _scipy_pattern(m.elements, m.n_dofs)
    B = spsp.coo_matrix((kl.ravel(), (r, c)), shape=(m.n_dofs,) * 2).tocsr()
    vals = np.zeros(p.nnz)
    for i in range(m.n_nodes):
        deg = p.nbr_ptr[i + 1] - p.nbr_ptr[i]
        for rr in range(deg):
            q = p.nbr_ptr[i] + rr
            srcs = blk_src[blk_ptr[q]:blk_ptr[q + 1]]
            assert np.all(np.diff(srcs // (npe * npe)) > 0)  # ascending element order
            for s in srcs:
                e, a, b = s // (npe * npe), (s // npe) % npe, s % npe
                assert m.elements[e, a] == i and m.elements[e, b] == p.nbr[q]
                blk = kl[e, 3 * a:3 * a + 3, 3 * b:3 * b + 3]
                for k in range(3):
                    o = 9 * p.nbr_ptr[i] + 3 * deg * k + 3 * rr
                    vals[o:o + 3] += blk[k]
    assert np.array_equal(vals, B.data)


def test_pattern_rejects_bad_connectivity():
    els = np.array([[0, 1, 2, 7]], dtype=np.int64)
    with pytest.raises(RuntimeError, match="invalid argument"):
        MeshPattern(els, 4)
    with pytest.raises(ValueError):
        MeshPattern(np.zeros((3, 5), dtype=np.int64), 8)


def test_fbar_plan_two_ring_and_volumetric_lists():
    """psx_fbar_plan_fill: two-ring lists and the common-neighbour lists of every block."""
    import ctypes

    from psierra_b200._lib import check, lib, ptr
    from psierra_b200.pattern import MeshPattern

    m = MESHES["unstructured"]()
    p = MeshPattern(m.elements, m.n_nodes)
    h = p.plan_host()
    N = m.n_nodes
    n2, nv = ctypes.c_int64(), ctypes.c_int64()
    check(lib().psx_fbar_plan_count(N, ptr(p.nbr_ptr), ptr(p.nbr), ctypes.byref(n2), ctypes.byref(nv)), "count")
    nbr2_ptr = np.zeros(N + 1, dtype=np.int32)
    nbr2 = np.zeros(int(n2.value), dtype=np.int32)
    pi2 = np.zeros(4 * h["n_pairs"], dtype=np.int32)
    ni2 = np.zeros(4 * N, dtype=np.int32)
    vptr = np.zeros(int(n2.value) + 1, dtype=np.int32)
    vsrc = np.zeros(3 * int(nv.value), dtype=np.int32)
    check(lib().psx_fbar_plan_fill(N, ptr(p.nbr_ptr), ptr(p.nbr), h["n_pairs"], ptr(h["pair_info"]), ptr(h["node_info"]),
                                   ptr(nbr2_ptr), ptr(nbr2), ptr(pi2), ptr(ni2), ptr(vptr), ptr(vsrc)), "fill")
    ring1 = [set(p.nbr[p.nbr_ptr[i]:p.nbr_ptr[i + 1]].tolist()) for i in range(N)]
    for b in range(N):
        want = sorted(set().union(*(ring1[a] for a in ring1[b])))
        got = nbr2[nbr2_ptr[b]:nbr2_ptr[b + 1]].tolist()
        assert got == want
        for t in range(nbr2_ptr[b], nbr2_ptr[b + 1]):
            c = int(nbr2[t])
            entries = vsrc[3 * vptr[t]:3 * vptr[t + 1]].reshape(-1, 3)
            assert entries[:, 0].tolist() == sorted(ring1[b] & ring1[c])
            for a, qab, qac in entries:
                assert p.nbr[qab] == b and p.nbr[qac] == c and p.nbr_ptr[a] <= qab < p.nbr_ptr[a + 1]
    assert int(nv.value) == sum(len(r) ** 2 for r in ring1)


@pytest.mark.parametrize("name", sorted(MESHES))
def test_nodal_csr_layout(name):
    """The assembler's pattern (and scipy's for the same mesh) is node-blocked, the layout
    PSX_PCG_NODAL asks for; a free-DOF slice or a reordered row is not."""
    from psierra_b200.solver import is_nodal_csr

    m = MESHES[name]()
    p = MeshPattern(m.elements, m.n_nodes)
    A, _, _ = _scipy_pattern(m.elements, m.n_dofs)
    assert is_nodal_csr(p.indptr, p.indices)
    assert is_nodal_csr(A.indptr, A.indices)
    free = np.arange(1, m.n_dofs)  # one DOF removed
    S = A[free][:, free].tocsr()
    assert not is_nodal_csr(S.indptr, S.indices)
    bad = p.indices.copy()
    r = int(np.argmax(np.diff(p.indptr) >= 6))  # a row with two neighbours or more
    a0 = p.indptr[r]
    bad[a0:a0 + 3], bad[a0 + 3:a0 + 6] = p.indices[a0 + 3:a0 + 6].copy(), p.indices[a0:a0 + 3].copy()
    assert not is_nodal_csr(p.indptr, bad)
