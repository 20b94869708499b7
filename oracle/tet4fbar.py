"""Tet4 F-bar element restated from psierra ``element/tet4_fbar.py``.  Test infrastructure only.

Nodal volume averaging (``tet4_fbar.py:17-33, 213-243``)::

    v0_a = sum_{e in E_a} V_e / 4,   v_a = sum_{e in E_a} V_e J_e / 4
    J_node_a = v_a / v0_a,           J_bar_e = mean_{a in e} J_node_a

Element (``tet4_fbar.py:147-211``): ratio = (J_bar / J)^(1/3), F_bar = ratio F,
(C, S_bar) = NeoHookean(F_bar), b_vol = (B_0 + B_1 + B_2) / 3, B_dev = B - m b_vol^T,
B_bar = ratio^2 B_dev + m b_vol^T, f = B_bar^T S_bar V,
k = B_bar^T C B_bar V + G^T (I (x) S_bar) G V.

Domain tangent (``tet4_fbar.py:355-459``): K = K_dev + K_vol with
K_dev = sum_e [ratio^4 B_dev^T (C - kappa m m^T) B_dev + G^T (I (x) S_bar) G] V and, per node a,
K_vol = kappa v0_a g_a g_a^T, g_a = sum_{e in E_a} (V_e J_e / (4 v0_a)) (B_0 + B_1 + B_2)_e on
the DOFs of a's element patch.  The sum K_dev + K_vol is scipy's CSR addition, which drops
entries that come out exactly zero.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as spsp

from oracle.assembly import assemble_sparse, assemble_vector, coo_indices, element_dofs
from oracle.neohookean import stress_and_tangent, stress_to_voigt
from oracle.tet4 import geometric_G, nonlinear_B, volume_and_gradients

M_VOIGT = np.array([1.0, 1.0, 1.0, 0.0, 0.0, 0.0])


def geometry(nodes, elements):
    """(H (E,4,3), V (E,), v0 (N,)) -- ``tet4_fbar.py:53-80``."""
    el = np.asarray(elements, dtype=np.int64)
    E = el.shape[0]
    H = np.zeros((E, 4, 3))
    V = np.zeros(E)
    for e in range(E):
        V[e], H[e] = volume_and_gradients(nodes[el[e]])
    v0 = np.bincount(el.ravel(), weights=np.repeat(0.25 * V, 4), minlength=nodes.shape[0])
    return H, V, v0


def jacobians(elements, u, H):
    """(F (E,3,3), J (E,)) with the inversion error of ``tet4_fbar.py:331-344``."""
    el = np.asarray(elements, dtype=np.int64)
    disp = np.asarray(u, dtype=np.float64).reshape(-1, 3)
    E = el.shape[0]
    F = np.zeros((E, 3, 3))
    J = np.zeros(E)
    for e in range(E):
        F[e] = np.eye(3) + disp[el[e]].T @ H[e]
        J[e] = np.linalg.det(F[e])
        if J[e] <= 0.0:
            raise ValueError(f"Element inversion detected at element {e}: det(F) = {J[e]:.4e} <= 0.")
    return F, J


def j_bar(elements, V, J, v0):
    el = np.asarray(elements, dtype=np.int64)
    v_node = np.bincount(el.ravel(), weights=np.repeat(0.25 * V * J, 4), minlength=v0.size)
    J_node = v_node / v0
    return J_node, np.mean(J_node[el], axis=1)


def element_force_and_tangent(X, u_nodes, mu, kappa, J_bar):
    """Single element with an explicit J_bar (``tet4_fbar.py:147-211``): (k 12x12, f 12)."""
    V, H = volume_and_gradients(X)
    l = u_nodes.T @ H
    F = np.eye(3) + l
    J = np.linalg.det(F)
    if J <= 0.0:
        raise ValueError(f"Element inversion detected: det(F) = {J:.4e} <= 0.")
    ratio = (J_bar / J) ** (1.0 / 3.0)
    C, S_bar = stress_and_tangent(ratio * F, mu, kappa)
    B = nonlinear_B(H, u_nodes)
    G = geometric_G(H)
    b_vol = (B[0] + B[1] + B[2]) / 3.0
    B_dev = B - np.outer(M_VOIGT, b_vol)
    B_bar = ratio ** 2 * B_dev + np.outer(M_VOIGT, b_vol)
    k = (B_bar.T @ C @ B_bar) * V + (G.T @ np.kron(np.eye(3), S_bar) @ G) * V
    f = (B_bar.T @ stress_to_voigt(S_bar)) * V
    return k, f


def internal_forces(nodes, elements, u, mu, kappa):
    """``Tet4Fbar.assemble_internal_forces`` (``tet4_fbar.py:248-312``)."""
    el = np.asarray(elements, dtype=np.int64)
    disp = np.asarray(u, dtype=np.float64).reshape(-1, 3)
    H, V, v0 = geometry(nodes, el)
    F, J = jacobians(el, disp, H)
    _, Jb = j_bar(el, V, J, v0)
    fl = np.zeros((el.shape[0], 12))
    for e in range(el.shape[0]):
        ratio = (Jb[e] / J[e]) ** (1.0 / 3.0)
        _, S_bar = stress_and_tangent(ratio * F[e], mu, kappa)
        B = nonlinear_B(H[e], disp[el[e]])
        b_vol = (B[0] + B[1] + B[2]) / 3.0
        B_bar = ratio ** 2 * (B - np.outer(M_VOIGT, b_vol)) + np.outer(M_VOIGT, b_vol)
        fl[e] = (B_bar.T @ stress_to_voigt(S_bar)) * V[e]
    return assemble_vector(fl, element_dofs(el), 3 * nodes.shape[0])


def tangent(nodes, elements, u, mu, kappa) -> spsp.csr_matrix:
    """``Tet4Fbar.assemble_tangent_stiffness_matrix`` (``tet4_fbar.py:314-459``)."""
    el = np.asarray(elements, dtype=np.int64)
    disp = np.asarray(u, dtype=np.float64).reshape(-1, 3)
    N, E = nodes.shape[0], el.shape[0]
    H, V, v0 = geometry(nodes, el)
    F, J = jacobians(el, disp, H)
    _, Jb = j_bar(el, V, J, v0)
    C_vol = kappa * np.outer(M_VOIGT, M_VOIGT)
    kd = np.zeros((E, 12, 12))
    div = np.zeros((E, 12))
    for e in range(E):
        ratio = (Jb[e] / J[e]) ** (1.0 / 3.0)
        C, S_bar = stress_and_tangent(ratio * F[e], mu, kappa)
        B = nonlinear_B(H[e], disp[el[e]])
        div[e] = B[0] + B[1] + B[2]
        B_dev = ratio ** 2 * (B - np.outer(M_VOIGT, div[e] / 3.0))
        G = geometric_G(H[e])
        kd[e] = (B_dev.T @ (C - C_vol) @ B_dev) * V[e] + (G.T @ np.kron(np.eye(3), S_bar) @ G) * V[e]
    ed = element_dofs(el)
    r, c = coo_indices(ed)
    K_dev = assemble_sparse(kd, r, c, 3 * N)
    # nodal volumetric blocks
    node_elems = [[] for _ in range(N)]
    for e in range(E):
        for a in el[e]:
            node_elems[a].append(e)
    rows, cols, vals = [], [], []
    for a in range(N):
        ea = np.array(node_elems[a], dtype=np.int64)
        if ea.size == 0:
            continue
        patch = np.unique(el[ea].ravel())
        dofs = np.repeat(patch * 3, 3) + np.tile(np.arange(3), patch.size)
        loc = {d: i for i, d in enumerate(dofs)}
        g = np.zeros(dofs.size)
        for e in ea:
            w = 0.25 * V[e] * J[e] / v0[a]
            for i, d in enumerate(ed[e]):
                g[loc[d]] += w * div[e, i]
        rr, cc = np.meshgrid(dofs, dofs, indexing="ij")
        rows.append(rr.ravel())
        cols.append(cc.ravel())
        vals.append(((kappa * v0[a]) * np.outer(g, g)).ravel())
    K_vol = spsp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                            shape=(3 * N, 3 * N)).tocsr()
    return K_dev + K_vol
