"""The gather plan (psx_plan_fill) emulated on the CPU.

Element records are built the way the element kernel writes them (off-diagonal block
of local pair (a < b) stored with rows = the node of smaller global id, diagonal
blocks as 6 values) from integer-valued element matrices, and gathered item by item
the way the gather kernel does; the result must equal scipy's COO->CSR of the same
element matrices exactly, and the granule ranges must hold exactly the items their
last contributing element makes ready.
"""
from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse as spsp

from oracle.assembly import coo_indices, element_dofs
from psierra_b200 import meshgen
from psierra_b200.pattern import MeshPattern
from test_pattern import MESHES


def _pairs(npe):
    return [(a, b) for a in range(npe) for b in range(a + 1, npe)]


def emulate(m, kl, fl, p: MeshPattern):
    E, npe = m.elements.shape
    h = p.plan_host()
    pairs = _pairs(npe)
    K = np.zeros(p.nnz)
    f = np.zeros(3 * m.n_nodes)
    gid = m.elements
    for q in range(h["n_pairs"]):
        pos_up, s_up, pos_lo, s_lo = h["pair_info"][4 * q:4 * q + 4]
        acc = np.zeros((3, 3))
        for src in h["pair_src"][h["pair_ptr"][q]:h["pair_ptr"][q + 1]]:
            e, slot = src >> 6, src & 63
            a, b = pairs[slot]
            blk = kl[e, 3 * a:3 * a + 3, 3 * b:3 * b + 3]
            acc += blk.T if gid[e, a] > gid[e, b] else blk
        for k in range(3):
            for mm in range(3):
                K[pos_up + s_up * k + mm] = acc[k, mm]
                K[pos_lo + s_lo * mm + k] = acc[k, mm]
    for q in range(m.n_nodes):
        pos, stride, node, _ = h["node_info"][4 * q:4 * q + 4]
        acc = np.zeros((3, 3))
        fa = np.zeros(3)
        for src in h["node_src"][h["node_ptr"][q]:h["node_ptr"][q + 1]]:
            e, a = src >> 4, src & 15
            acc += kl[e, 3 * a:3 * a + 3, 3 * a:3 * a + 3]
            fa += fl[e, 3 * a:3 * a + 3]
        if stride > 0:
            for k in range(3):
                K[pos + stride * k: pos + stride * k + 3] = acc[k]
        f[3 * node:3 * node + 3] = fa
    return K, f


@pytest.mark.parametrize("name", ["cfg1", "unstructured", "tet10", "single"])
def test_plan_gather_reproduces_coo_sum(name):
    m = MESHES[name]()
    p = MeshPattern(m.elements, m.n_nodes)
    E, npe = m.elements.shape
    rng = np.random.default_rng(3)
    kl = rng.integers(-1000, 1000, size=(E, 3 * npe, 3 * npe)).astype(np.float64)
    kl = kl + np.transpose(kl, (0, 2, 1))  # element tangents are symmetric
    fl = rng.integers(-1000, 1000, size=(E, 3 * npe)).astype(np.float64)
    K, f = emulate(m, kl, fl, p)
    ed = element_dofs(m.elements)
    r, c = coo_indices(ed)
    B = spsp.coo_matrix((kl.ravel(), (r, c)), shape=(m.n_dofs,) * 2).tocsr()
    fr = np.zeros(m.n_dofs)
    np.add.at(fr, ed.ravel(), fl.ravel())
    assert np.array_equal(K, B.data)
    assert np.array_equal(f, fr)


def test_plan_granules_and_span():
    m = meshgen.box_tet4(1.0, 1.0, 1.0, 12, 10, 9)
    p = MeshPattern(m.elements, m.n_nodes)
    p.granule = 256
    h = p.plan_host()
    g = p.granule
    span = int(h["max_span"][0])
    for q in range(h["n_pairs"]):
        es = h["pair_src"][h["pair_ptr"][q]:h["pair_ptr"][q + 1]] >> 6
        assert np.all(np.diff(es) > 0)
        gr = int(np.searchsorted(h["pair_gptr"], q, side="right") - 1)
        assert gr * g <= es.max() < (gr + 1) * g
        assert es.max() - es.min() <= span
    for q in range(m.n_nodes):
        es = h["node_src"][h["node_ptr"][q]:h["node_ptr"][q + 1]] >> 4
        gr = int(np.searchsorted(h["node_gptr"], q, side="right") - 1)
        assert gr * g <= es.max() < (gr + 1) * g
        assert es.max() - es.min() <= span
    assert h["pair_gptr"][-1] == h["n_pairs"] and h["node_gptr"][-1] == m.n_nodes
