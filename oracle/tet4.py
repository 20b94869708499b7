"""Tet4 Total-Lagrangian element restated from psierra ``element/tet4_base.py`` and
``element/tet4_total_lagrangian.py``.  Test infrastructure only."""
from __future__ import annotations

import numpy as np

from oracle.neohookean import constitutive_matrix, stress_and_tangent, stress_to_voigt


def volume_and_gradients(X: np.ndarray) -> tuple[float, np.ndarray]:
    """``tet4_base.py:34-67``: A=[1 X], V=det(A)/6, H=(A^-1)[1:,:]^T."""
    A = np.ones((4, 4), dtype=np.float64)
    A[:, 1:] = X
    detA = np.linalg.det(A)
    if detA <= 0.0:
        raise ValueError(
            f"Negative or zero element volume detected (det(A) = {detA}). "
            "Check element vertex ordering.")
    return detA / 6.0, np.linalg.inv(A)[1:, :].T


def linear_B(H: np.ndarray) -> np.ndarray:
    """``tet4_base.py:73-95`` (Voigt xx,yy,zz,xy,yz,zx with engineering shear)."""
    n = H.shape[0]
    BL = np.zeros((6, 3 * n), dtype=np.float64)
    for i in range(n):
        b, c, d = H[i]
        col = 3 * i
        BL[0, col] = b
        BL[1, col + 1] = c
        BL[2, col + 2] = d
        BL[3, col], BL[3, col + 1] = c, b
        BL[4, col + 1], BL[4, col + 2] = d, c
        BL[5, col], BL[5, col + 2] = d, b
    return BL


def geometric_G(H: np.ndarray) -> np.ndarray:
    """``tet4_base.py:97-123``: 9 x 3n map to the displacement gradient."""
    n = H.shape[0]
    G = np.zeros((9, 3 * n), dtype=np.float64)
    for i in range(n):
        for comp in range(3):
            G[3 * comp:3 * comp + 3, 3 * i + comp] = H[i]
    return G


def nonlinear_B(H: np.ndarray, u: np.ndarray) -> np.ndarray:
    """``tet4_total_lagrangian.py:24-75``: B = B_L + B_NL(l), l = u^T H."""
    n = H.shape[0]
    l = u.T @ H
    du, dv, dw = l[0], l[1], l[2]
    BNL = np.zeros((6, 3 * n), dtype=np.float64)
    for i in range(n):
        b, c, d = H[i]
        col = 3 * i
        BNL[0, col:col + 3] = du[0] * b, dv[0] * b, dw[0] * b
        BNL[1, col:col + 3] = du[1] * c, dv[1] * c, dw[1] * c
        BNL[2, col:col + 3] = du[2] * d, dv[2] * d, dw[2] * d
        BNL[3, col:col + 3] = du[0] * c + du[1] * b, dv[0] * c + dv[1] * b, dw[0] * c + dw[1] * b
        BNL[4, col:col + 3] = du[1] * d + du[2] * c, dv[1] * d + dv[2] * c, dw[1] * d + dw[2] * c
        BNL[5, col:col + 3] = du[0] * d + du[2] * b, dv[0] * d + dv[2] * b, dw[0] * d + dw[2] * b
    return linear_B(H) + BNL


def force_and_tangent(X: np.ndarray, u: np.ndarray, mu: float, kappa: float):
    """``tet4_total_lagrangian.py:77-139``: returns (k_tan 12x12, f_int 12)."""
    V, H = volume_and_gradients(X)
    x = X + u
    F = x.T @ H
    J = np.linalg.det(F)
    if J <= 0.0:
        raise ValueError(f"Element inversion detected: det(F) = {J:.4e} <= 0.")
    C, S = stress_and_tangent(F, mu, kappa)
    B = nonlinear_B(H, u)
    G = geometric_G(H)
    k_mat = (B.T @ C @ B) * V
    k_geo = (G.T @ np.kron(np.identity(3), S) @ G) * V
    f = (B.T @ stress_to_voigt(S)) * V
    return k_mat + k_geo, f


def linear_stiffness(X: np.ndarray, lam: float, mu: float) -> np.ndarray:
    """``tet4_base.py:129-136``: k_e = B_L^T C B_L V with the small-strain C."""
    V, H = volume_and_gradients(X)
    BL = linear_B(H)
    return (BL.T @ constitutive_matrix(lam, mu) @ BL) * V


def mass_matrix(rho: float, volume: float) -> np.ndarray:
    """``tet4_base.py:138-151``: consistent mass, weight 2 on the diagonal blocks."""
    f = rho * volume / 20.0
    m = np.zeros((12, 12))
    for i in range(4):
        for j in range(4):
            m[3 * i:3 * i + 3, 3 * j:3 * j + 3] = (2.0 if i == j else 1.0) * f * np.identity(3)
    return m
