"""Host side of the two-level preconditioner (CPU): aggregation, the distance-2
colouring, and the probing scatter that assembles A_c = P^T A P, against a dense
restatement of P; and the preconditioner's action against its definition."""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import torch

from oracle.vectorized import assemble_force_and_tangent
from psierra_b200 import meshgen
from psierra_b200.coarse import CoarseSpace, aggregate_graph, distance2_colouring, slice_aggregates


def _beams():
    meshes = [meshgen.box_tet4(0.6, 0.1, 0.1, 24, 3, 3), meshgen.box_tet4(0.1, 0.5, 0.1, 3, 20, 3)]
    union, node_off, _ = meshgen.concat_meshes(meshes)
    return meshes, union, node_off


def _dense_P(X, node_agg, fixed, n_agg):
    """Column 6a + s of P: translations e_s, rotations e_(s-3) x (X_i - c_a); zero rows on
    fixed DOFs."""
    N = X.shape[0]
    cent = np.zeros((n_agg, 3))
    np.add.at(cent, node_agg, X)
    cent /= np.bincount(node_agg, minlength=n_agg)[:, None]
    P = np.zeros((3 * N, 6 * n_agg))
    for i in range(N):
        a = node_agg[i]
        d = X[i] - cent[a]
        for s in range(3):
            P[3 * i + s, 6 * a + s] = 1.0
        for e in range(3):
            ev = np.zeros(3)
            ev[e] = 1.0
            P[3 * i:3 * i + 3, 6 * a + 3 + e] = np.cross(ev, d)
    P[np.asarray(fixed, dtype=bool)] = 0.0
    return P


def test_slices_follow_the_long_axis_and_colouring_is_distance_two():
    meshes, union, node_off = _beams()
    node_agg, block_agg = slice_aggregates(union.nodes, node_off, levels_per_aggregate=2)
    assert block_agg[0] == 0 and np.all(np.diff(block_agg) > 1)
    for b, m in enumerate(meshes):
        agg = node_agg[node_off[b]:node_off[b + 1]]
        assert agg.min() == block_agg[b] and agg.max() == block_agg[b + 1] - 1
        axis = int(np.argmax(np.ptp(m.nodes, axis=0)))
        # a slice holds whole cross-sections: equal coordinates along the axis share it
        for x in np.unique(m.nodes[:, axis]):
            assert len(np.unique(agg[m.nodes[:, axis] == x])) == 1
    n_agg = int(block_agg[-1])
    ptr_, nbr = aggregate_graph(union.elements, node_agg, n_agg)
    colour = distance2_colouring(ptr_, nbr)
    for b in range(n_agg):
        nb = nbr[ptr_[b]:ptr_[b + 1]]
        assert b in nb
        assert len(np.unique(colour[nb])) == len(nb)  # no colour twice around b


def test_probing_assembles_P_T_A_P_and_the_preconditioner_matches_its_definition():
    meshes, union, node_off = _beams()
    mu, _, kappa = meshgen.lame_from_young_poisson(1e5, 0.3)
    u = 1e-4 * np.random.default_rng(3).standard_normal(union.nodes.shape)
    _, K = assemble_force_and_tangent(union.nodes, union.elements, u, mu, kappa)
    fixed = np.zeros(3 * union.n_nodes, dtype=np.uint8)
    for b, m in enumerate(meshes):
        axis = int(np.argmax(np.ptp(m.nodes, axis=0)))
        clamp = node_off[b] + meshgen.nodes_on_plane(m, axis, "min")
        fixed[np.concatenate([3 * clamp + c for c in range(3)])] = 1
    # symmetric elimination, as psx_csr_dirichlet does it
    keep = sp.diags((fixed == 0).astype(float))
    K = (keep @ K @ keep + sp.diags(fixed.astype(float))).tocsr()
    cs = CoarseSpace(union.nodes, union.elements, fixed, node_off, levels_per_aggregate=2, device="cpu")
    node_agg = cs.node_agg.numpy().astype(np.int64)
    P = _dense_P(union.nodes, node_agg, fixed, cs.n_agg)
    colour = cs.agg_colour.numpy()
    for c in range(cs.n_colours):
        for s in range(6):
            v = P[:, 6 * np.where(colour == c)[0] + s].sum(axis=1)
            cs.fill(c, s, torch.from_numpy(P.T @ (K @ v)))
    Ac = P.T @ K @ P
    ba = cs.block_agg.numpy()
    for b in range(cs.n_blocks):
        sl = slice(6 * ba[b], 6 * ba[b + 1])
        m = 6 * (ba[b + 1] - ba[b])
        got = cs.ac[b, :m, :m].numpy()
        assert np.abs(got - Ac[sl, sl]).max() <= 1e-12 * np.abs(Ac[sl, sl]).max()
    assert np.abs(Ac[:6 * ba[1], 6 * ba[1]:]).max() == 0.0  # instances are uncoupled
    cs.invert()
    assert bool(cs.factor_ok.all())
    r = np.random.default_rng(4).standard_normal(3 * union.n_nodes) * (fixed == 0)
    rc = P.T @ r
    yc = np.zeros_like(rc)
    for b in range(cs.n_blocks):
        sl = slice(6 * ba[b], 6 * ba[b + 1])
        m = 6 * (ba[b + 1] - ba[b])
        yc[sl] = cs.ainv[b, :m, :m].numpy() @ rc[sl]
        want = np.linalg.solve(Ac[sl, sl] + 1e-12 * np.abs(np.diag(Ac[sl, sl])).max() * np.eye(m), rc[sl])
        assert np.abs(yc[sl] - want).max() <= 1e-8 * np.abs(want).max()
