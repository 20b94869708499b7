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


def tile_meta(h, T, t):
    """(np, nn, pair offsets, node offsets, pair codes, node codes) of tile t."""
    m = h["tile_meta"][t * h["tile_meta_stride"]:(t + 1) * h["tile_meta_stride"]].astype(np.int64)
    up4 = lambda b: (b + 3) // 4 * 4  # noqa: E731
    off_n = 4
    src_n = off_n + up4(4 * T + 1)
    off_p = src_n + 4 * T
    src_p = off_p + up4(6 * T + 1)
    n_p, n_n = int(m[0]), int(m[1])
    return (n_p, n_n, m[off_p:off_p + n_p + 1], m[off_n:off_n + n_n + 1], m[src_p:src_p + 6 * T],
            m[src_n:src_n + 4 * T])


def emulate_tiles(m, kl, fl, p: MeshPattern):
    """Tile records (psx_tile_plan_fill) summed per tile, then gathered per item."""
    E = m.n_elements
    h = p.plan_host()
    T = p.tile
    pairs = _pairs(4)
    gid = m.elements
    cap_p, cap_n = (int(c) for c in h["tile_caps"])
    nt = (E + T - 1) // T
    rec_p = np.zeros((nt, cap_p, 3, 3))
    rec_d = np.zeros((nt, cap_n, 3, 3))
    rec_f = np.zeros((nt, cap_n, 3))
    for t in range(nt):
        n_p, n_n, offp, offn, srcp, srcn = tile_meta(h, T, t)
        for lp in range(n_p):
            for c in srcp[offp[lp]:offp[lp + 1]]:
                e, s = t * T + (c >> 3), c & 7
                a, b = pairs[s]
                blk = kl[e, 3 * a:3 * a + 3, 3 * b:3 * b + 3]
                rec_p[t, lp] += blk.T if gid[e, a] > gid[e, b] else blk
        for ln in range(n_n):
            for c in srcn[offn[ln]:offn[ln + 1]]:
                e, a = t * T + (c >> 2), c & 3
                rec_d[t, ln] += kl[e, 3 * a:3 * a + 3, 3 * a:3 * a + 3]
                rec_f[t, ln] += fl[e, 3 * a:3 * a + 3]
    K = np.zeros(p.nnz)
    f = np.zeros(3 * m.n_nodes)
    for q in range(h["n_pairs"]):
        pos_up, s_up, pos_lo, s_lo = h["pair_info"][4 * q:4 * q + 4]
        acc = np.zeros((3, 3))
        for c in h["pair_src_t"][h["pair_ptr_t"][q]:h["pair_ptr_t"][q + 1]]:
            acc += rec_p[c >> 8, c & 255]
        for k in range(3):
            for mm in range(3):
                K[pos_up + s_up * k + mm] = acc[k, mm]
                K[pos_lo + s_lo * mm + k] = acc[k, mm]
    for q in range(m.n_nodes):
        pos, stride, node, _ = h["node_info"][4 * q:4 * q + 4]
        acc = np.zeros((3, 3))
        fa = np.zeros(3)
        for c in h["node_src_t"][h["node_ptr_t"][q]:h["node_ptr_t"][q + 1]]:
            acc += rec_d[c >> 7, c & 127]
            fa += rec_f[c >> 7, c & 127]
        if stride > 0:
            for k in range(3):
                K[pos + stride * k: pos + stride * k + 3] = acc[k]
        f[3 * node:3 * node + 3] = fa
    return K, f, h


@pytest.mark.parametrize("name", ["cfg1", "unstructured", "single"])
def test_tile_plan_gather_reproduces_coo_sum(name):
    m = MESHES[name]()
    p = MeshPattern(m.elements, m.n_nodes)
    E = m.n_elements
    rng = np.random.default_rng(5)
    kl = rng.integers(-1000, 1000, size=(E, 12, 12)).astype(np.float64)
    kl = kl + np.transpose(kl, (0, 2, 1))
    fl = rng.integers(-1000, 1000, size=(E, 12)).astype(np.float64)
    K, f, h = emulate_tiles(m, kl, fl, p)
    ed = element_dofs(m.elements)
    r, c = coo_indices(ed)
    B = spsp.coo_matrix((kl.ravel(), (r, c)), shape=(m.n_dofs,) * 2).tocsr()
    fr = np.zeros(m.n_dofs)
    np.add.at(fr, ed.ravel(), fl.ravel())
    assert np.array_equal(K, B.data)
    assert np.array_equal(f, fr)
    # every element slot appears exactly once in its tile's lists; codes ascend within
    # a local pair; gather lists ascend by tile (fixed summation order)
    T = p.tile
    assert h["tile_meta_stride"] % 16 == 0
    for t in range((E + T - 1) // T):
        n = min(T, E - t * T)
        n_p, n_n, off, offn, codes, codesn = tile_meta(h, T, t)
        assert off[-1] == 6 * n and offn[-1] == 4 * n
        assert sorted(codes[:6 * n].tolist()) == sorted(el * 8 + s for el in range(n) for s in range(6))
        assert sorted(codesn[:4 * n].tolist()) == sorted(el * 4 + a for el in range(n) for a in range(4))
        for lp in range(n_p):
            assert np.all(np.diff(codes[off[lp]:off[lp + 1]]) > 0)
    for q in range(h["n_pairs"]):
        tiles = h["pair_src_t"][h["pair_ptr_t"][q]:h["pair_ptr_t"][q + 1]] >> 8
        assert np.all(np.diff(tiles) > 0)
    assert h["tile_caps"][0] <= 6 * T and h["tile_caps"][1] <= 4 * T
