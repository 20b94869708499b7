"""NeoHookean material restated from psierra ``material/neohookean.py``.

Test infrastructure only (see ``oracle/__init__.py``).
"""
from __future__ import annotations

import numpy as np

# psierra utility/tensor.py:5-12 (xx, yy, zz, xy, yz, zx)
VOIGT_MAP_3D = {0: (0, 0), 1: (1, 1), 2: (2, 2), 3: (0, 1), 4: (1, 2), 5: (2, 0)}


def constitutive_matrix(lam: float, mu: float) -> np.ndarray:
    """Small-strain 6x6 isotropic matrix; psierra ``material/neohookean.py:33-53``."""
    C = np.zeros((6, 6), dtype=np.float64)
    c11 = lam + 2.0 * mu
    C[0, 0] = C[1, 1] = C[2, 2] = c11
    C[0, 1] = C[1, 0] = C[0, 2] = C[2, 0] = C[1, 2] = C[2, 1] = lam
    C[3, 3] = C[4, 4] = C[5, 5] = mu
    return C


def stress_and_tangent(F: np.ndarray, mu: float, kappa: float) -> tuple[np.ndarray, np.ndarray]:
    """(C_voigt 6x6, S 3x3) for ``Psi = mu/2 (J^-2/3 I1 - 3) + K/2 (ln J)^2``.

    Restates psierra ``material/neohookean.py:55-122`` step for step: LAPACK
    ``det``/``inv``, the five ``einsum`` outer products, Voigt extraction.
    """
    J = float(np.linalg.det(F))
    if J <= 0.0:  # neohookean.py:75-77
        raise ValueError(f"Element inversion detected: det(F) = {J:.4e} <= 0.")
    C = F.T @ F  # :79
    C_inv = np.linalg.inv(C)  # :80
    I1 = float(np.trace(C))  # :81
    I3 = np.identity(3, dtype=np.float64)
    factor = mu * (J ** (-2.0 / 3.0))  # :87
    S = factor * (I3 - (1.0 / 3.0) * I1 * C_inv) + kappa * np.log(J) * C_inv  # :90-92
    C_inv_outer = np.einsum("ij,kl->ijkl", C_inv, C_inv)  # :95
    I_Cinv = 0.5 * (np.einsum("ik,jl->ijkl", C_inv, C_inv) + np.einsum("il,jk->ijkl", C_inv, C_inv))
    C4_vol = kappa * C_inv_outer - 2.0 * kappa * np.log(J) * I_Cinv  # :102
    C_inv_I = np.einsum("ij,kl->ijkl", C_inv, I3) + np.einsum("ij,kl->ijkl", I3, C_inv)
    C4_iso = (-(2.0 / 3.0) * factor * C_inv_I + (2.0 / 9.0) * factor * I1 * C_inv_outer
              + (2.0 / 3.0) * factor * I1 * I_Cinv)  # :108-112
    C4 = C4_vol + C4_iso
    Cv = np.zeros((6, 6), dtype=np.float64)
    for a, (i, j) in VOIGT_MAP_3D.items():  # :117-120
        for b, (k, l) in VOIGT_MAP_3D.items():
            Cv[a, b] = C4[i, j, k, l]
    return Cv, S


def stress_to_voigt(S: np.ndarray) -> np.ndarray:
    """psierra ``utility/tensor.py:15-38``."""
    return np.array([S[0, 0], S[1, 1], S[2, 2], S[0, 1], S[1, 2], S[2, 0]], dtype=np.float64)
