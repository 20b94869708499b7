"""Batched (all elements at once) numpy form of the same Tet4/Tet10 algorithm.

Test infrastructure only.  It evaluates the identical formulas as
``oracle.tet4.force_and_tangent`` / ``oracle.tet10.force_and_tangent`` (B^T C B,
G^T (I x S) G, B^T S_voigt, psierra ``element/tet4_total_lagrangian.py:77-139``,
``element/tet10_total_lagrangian.py:63-136``, ``material/neohookean.py:55-122``)
with ``einsum`` over the element axis, so parity checks at tens of thousands of
elements finish in seconds.  ``tests/test_oracle_golden.py`` checks it against the
per-element restatement and against the reference's own outputs.
"""
from __future__ import annotations

import numpy as np

from oracle.tet10 import quadrature4, shape_gradients_ref

_VOIGT = [(0, 0), (1, 1), (2, 2), (0, 1), (1, 2), (2, 0)]


def _material(F, mu, kappa):
    """Batched ``NeoHookean.compute_stress_and_tangent`` -> (C_voigt (n,6,6), S (n,3,3), J)."""
    J = np.linalg.det(F)
    C = np.einsum("nki,nkj->nij", F, F)
    Ci = np.linalg.inv(C)
    I1 = np.einsum("nii->n", C)
    I3 = np.identity(3)
    fac = mu * J ** (-2.0 / 3.0)
    lnJ = np.log(np.where(J > 0, J, 1.0))
    S = fac[:, None, None] * (I3 - (I1 / 3.0)[:, None, None] * Ci) + (kappa * lnJ)[:, None, None] * Ci
    Cv = np.zeros((F.shape[0], 6, 6))
    for a, (i, j) in enumerate(_VOIGT):
        for b, (k, l) in enumerate(_VOIGT):
            outer = Ci[:, i, j] * Ci[:, k, l]
            isym = 0.5 * (Ci[:, i, k] * Ci[:, j, l] + Ci[:, i, l] * Ci[:, j, k])
            cI = Ci[:, i, j] * I3[k, l] + I3[i, j] * Ci[:, k, l]
            Cv[:, a, b] = (kappa * outer - 2.0 * kappa * lnJ * isym
                           - (2.0 / 3.0) * fac * cI + (2.0 / 9.0) * fac * I1 * outer
                           + (2.0 / 3.0) * fac * I1 * isym)
    return Cv, S, J


def _B_matrices(H, F):
    """Batched B(u) (n,6,3m) = Voigt rows of F^T grad N; H is (n, m, 3)."""
    n, m, _ = H.shape
    B = np.zeros((n, 6, 3 * m))
    for a in range(m):
        for k in range(3):
            col = 3 * a + k
            for r, (i, j) in enumerate(_VOIGT):
                if i == j:
                    B[:, r, col] = F[:, k, i] * H[:, a, i]
                else:
                    B[:, r, col] = F[:, k, i] * H[:, a, j] + F[:, k, j] * H[:, a, i]
    return B


def _qp_contrib(H, w, x, mu, kappa):
    F = np.einsum("nak,naj->nkj", x, H)
    Cv, S, J = _material(F, mu, kappa)
    if np.any(J <= 0):
        e = int(np.argmax(J <= 0))
        raise ValueError(f"Element inversion detected: det(F) = {J[e]:.4e} <= 0.")
    B = _B_matrices(H, F)
    kmat = np.einsum("nri,nrs,nsj->nij", B, Cv, B)
    HSH = np.einsum("nai,nij,nbj->nab", H, S, H)
    m = H.shape[1]
    kgeo = np.einsum("nab,kl->nakbl", HSH, np.identity(3)).reshape(-1, 3 * m, 3 * m)
    Sv = np.stack([S[:, i, j] for (i, j) in _VOIGT], axis=1)
    f = np.einsum("nri,nr->ni", B, Sv)
    return (kmat + kgeo) * w[:, None, None], f * w[:, None]


def element_force_and_tangent(nodes, elements, u, mu, kappa):
    """(k (E,d,d), f (E,d)) for all elements; mu/kappa scalar or (E,)."""
    el = np.asarray(elements, dtype=np.int64)
    E, npe = el.shape
    mu = np.broadcast_to(np.asarray(mu, dtype=np.float64), (E,))
    kappa = np.broadcast_to(np.asarray(kappa, dtype=np.float64), (E,))
    X = nodes[el]
    x = X + u[el]
    if npe == 4:
        A = np.ones((E, 4, 4))
        A[:, :, 1:] = X
        detA = np.linalg.det(A)
        H = np.transpose(np.linalg.inv(A)[:, 1:, :], (0, 2, 1))
        return _qp_contrib(H, detA / 6.0, x, mu, kappa)
    qp, qw = quadrature4()
    k = np.zeros((E, 30, 30))
    f = np.zeros((E, 30))
    for q in range(4):
        dN = shape_gradients_ref(*qp[q])
        Jm = np.einsum("nai,aj->nij", X, dN)
        detJ = np.linalg.det(Jm)
        H = np.einsum("aj,nji->nai", dN, np.linalg.inv(Jm))
        kq, fq = _qp_contrib(H, qw[q] * detJ, x, mu, kappa)
        k += kq
        f += fq
    return k, f


def assemble_force_and_tangent(nodes, elements, u, mu, kappa):
    from oracle.assembly import assemble_sparse, assemble_vector, coo_indices, element_dofs

    k, f = element_force_and_tangent(nodes, elements, u, mu, kappa)
    ed = element_dofs(elements)
    r, c = coo_indices(ed)
    n = 3 * nodes.shape[0]
    return assemble_vector(f, ed, n), assemble_sparse(k, r, c, n)
