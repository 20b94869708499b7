"""Tet10 Total-Lagrangian element restated from psierra ``element/tet10_base.py``,
``element/tet10_total_lagrangian.py`` and ``element/quadrature.py``.
Test infrastructure only."""
from __future__ import annotations

import numpy as np

from oracle.neohookean import constitutive_matrix, stress_and_tangent, stress_to_voigt
from oracle.tet4 import geometric_G, linear_B, nonlinear_B


def quadrature4():
    """``quadrature.py:36-49``: a=(5-sqrt5)/20, b=(5+3sqrt5)/20, w=1/24."""
    a = (5.0 - np.sqrt(5.0)) / 20.0
    b = (5.0 + 3.0 * np.sqrt(5.0)) / 20.0
    qp = np.array([[a, a, a], [b, a, a], [a, b, a], [a, a, b]], dtype=np.float64)
    return qp, np.full(4, 1.0 / 24.0)


def shape_gradients_ref(xi: float, eta: float, zeta: float) -> np.ndarray:
    """``tet10_base.py:118-179`` (VTK ordering)."""
    L1, L2, L3 = xi, eta, zeta
    L0 = 1.0 - L1 - L2 - L3
    dN = np.zeros((10, 3))
    dN[0, :] = -(4.0 * L0 - 1.0)
    dN[1, 0] = 4.0 * L1 - 1.0
    dN[2, 1] = 4.0 * L2 - 1.0
    dN[3, 2] = 4.0 * L3 - 1.0
    dN[4] = [4.0 * (L0 - L1), -4.0 * L1, -4.0 * L1]
    dN[5] = [4.0 * L2, 4.0 * L1, 0.0]
    dN[6] = [-4.0 * L2, 4.0 * (L0 - L2), -4.0 * L2]
    dN[7] = [-4.0 * L3, -4.0 * L3, 4.0 * (L0 - L3)]
    dN[8] = [4.0 * L3, 0.0, 4.0 * L1]
    dN[9] = [0.0, 4.0 * L3, 4.0 * L2]
    return dN


def force_and_tangent(X: np.ndarray, u: np.ndarray, mu: float, kappa: float):
    """``tet10_total_lagrangian.py:63-136``: (k_tan 30x30, f_int 30)."""
    qp, qw = quadrature4()
    x = X + u
    k = np.zeros((30, 30))
    f = np.zeros(30)
    for q in range(4):
        dN = shape_gradients_ref(*qp[q])
        Jm = X.T @ dN
        detJ = np.linalg.det(Jm)
        if detJ <= 0.0:
            raise ValueError(f"Negative or zero Jacobian determinant: det(J) = {detJ:.4e}.")
        H = dN @ np.linalg.inv(Jm)
        F = x.T @ H
        detF = np.linalg.det(F)
        if detF <= 0.0:
            raise ValueError(f"Element inversion detected: det(F) = {detF:.4e} <= 0.")
        C, S = stress_and_tangent(F, mu, kappa)
        B = nonlinear_B(H, u)
        G = geometric_G(H)
        w = qw[q] * detJ
        k += (B.T @ C @ B + G.T @ np.kron(np.identity(3), S) @ G) * w
        f += (B.T @ stress_to_voigt(S)) * w
    return k, f


def linear_stiffness(X: np.ndarray, lam: float, mu: float) -> np.ndarray:
    """``tet10_base.py:310-342``."""
    qp, qw = quadrature4()
    C = constitutive_matrix(lam, mu)
    k = np.zeros((30, 30))
    for q in range(4):
        dN = shape_gradients_ref(*qp[q])
        Jm = X.T @ dN
        detJ = np.linalg.det(Jm)
        H = dN @ np.linalg.inv(Jm)
        BL = linear_B(H)
        k += qw[q] * (BL.T @ C @ BL) * detJ
    return k
