"""Material parameters and the NeoHookean material, mirroring pSierra's API.

``IsotropicElasticParameters`` and ``NeoHookean`` keep the names, setters and
derived moduli of psierra ``material/parameters.py:6-140`` and
``material/neohookean.py:9-53`` so code written against the reference builds the
same objects.  The GPU element reads ``parameters.shear_modulus``,
``parameters.bulk_modulus`` and ``parameters.lame_parameter_1`` -- it accepts the
reference's own material objects as well.

``NeoHookeanField`` adds what the reference lacks: per-element shear and bulk
moduli (``mu_e``, ``kappa_e``), used by batched multi-instance meshes and by the
adjoint parameter identification.  A reference ``NeoHookean`` is the special case of
a constant field.
"""
from __future__ import annotations

import numpy as np


class IsotropicElasticParameters:
    """Isotropic elastic moduli; setters follow psierra ``material/parameters.py:43-140``."""

    def __init__(self) -> None:
        self._youngs_modulus = None
        self._poissons_ratio = None
        self._shear_modulus = None
        self._lame_parameter_1 = None
        self._lame_parameter_2 = None
        self._bulk_modulus = None
        self._p_wave_modulus = None
        self._mass_density = None

    @staticmethod
    def _validate_density(rho: float) -> None:
        if rho <= 0.0:
            raise ValueError(f"Mass density must be positive. Got {rho}")

    def set_from_youngs_poisson(self, youngs_modulus: float, poissons_ratio: float, mass_density: float) -> None:
        E, nu, rho = float(youngs_modulus), float(poissons_ratio), float(mass_density)
        if E <= 0.0:
            raise ValueError(f"Young's modulus must be positive. Got {E}")
        if not (-1.0 < nu < 0.5):
            raise ValueError(f"Poisson's ratio must satisfy -1.0 < poissons_ratio < 0.5. Got {nu}")
        self._validate_density(rho)
        self._youngs_modulus, self._poissons_ratio, self._mass_density = E, nu, rho
        mu = E / (2.0 * (1.0 + nu))
        lam = (E * nu) / ((1.0 + nu) * (1.0 - 2.0 * nu))
        kappa = E / (3.0 * (1.0 - 2.0 * nu))
        self._shear_modulus = self._lame_parameter_2 = mu
        self._lame_parameter_1 = lam
        self._bulk_modulus = kappa
        self._p_wave_modulus = lam + 2.0 * mu

    def set_from_bulk_shear(self, bulk_modulus: float, shear_modulus: float, mass_density: float) -> None:
        kappa, mu, rho = float(bulk_modulus), float(shear_modulus), float(mass_density)
        if kappa <= 0.0:
            raise ValueError(f"Bulk modulus must be positive. Got {kappa}")
        if mu <= 0.0:
            raise ValueError(f"Shear modulus must be positive. Got {mu}")
        self._validate_density(rho)
        self._bulk_modulus, self._shear_modulus, self._lame_parameter_2 = kappa, mu, mu
        self._mass_density = rho
        self._lame_parameter_1 = kappa - (2.0 / 3.0) * mu
        self._youngs_modulus = (9.0 * kappa * mu) / (3.0 * kappa + mu)
        self._poissons_ratio = (3.0 * kappa - 2.0 * mu) / (2.0 * (3.0 * kappa + mu))
        self._p_wave_modulus = kappa + (4.0 / 3.0) * mu

    def set_from_lame_parameters(self, lame_parameter_1: float, lame_parameter_2: float, mass_density: float) -> None:
        lam, mu, rho = float(lame_parameter_1), float(lame_parameter_2), float(mass_density)
        if mu <= 0.0:
            raise ValueError(f"Lamé parameter 2 (shear modulus) must be positive. Got {mu}")
        if (lam + mu) <= 0.0:
            raise ValueError(
                f"Constraint (lame_parameter_1 + lame_parameter_2 > 0) violated. Got lambda={lam}, mu={mu}")
        self._validate_density(rho)
        self._lame_parameter_1, self._lame_parameter_2, self._shear_modulus = lam, mu, mu
        self._mass_density = rho
        self._bulk_modulus = lam + (2.0 / 3.0) * mu
        self._youngs_modulus = (mu * (3.0 * lam + 2.0 * mu)) / (lam + mu)
        self._poissons_ratio = lam / (2.0 * (lam + mu))
        self._p_wave_modulus = lam + 2.0 * mu

    @property
    def youngs_modulus(self):
        return self._youngs_modulus

    @property
    def poissons_ratio(self):
        return self._poissons_ratio

    @property
    def shear_modulus(self):
        return self._shear_modulus

    @property
    def lame_parameter_1(self):
        return self._lame_parameter_1

    @property
    def lame_parameter_2(self):
        return self._lame_parameter_2

    @property
    def bulk_modulus(self):
        return self._bulk_modulus

    @property
    def p_wave_modulus(self):
        return self._p_wave_modulus

    @property
    def mass_density(self):
        return self._mass_density


class NeoHookean:
    """Compressible NeoHookean, ``Psi = mu/2 (J^-2/3 I1 - 3) + K/2 (ln J)^2``
    (psierra ``material/neohookean.py:9-122``).  Stress and tangent are evaluated
    inside the element kernels; this object carries the parameters."""

    def __init__(self, parameters: IsotropicElasticParameters) -> None:
        self._parameters = parameters

    @property
    def parameters(self) -> IsotropicElasticParameters:
        return self._parameters

    @property
    def mass_density(self) -> float:
        return self._parameters.mass_density

    def compute_constitutive_matrix(self) -> np.ndarray:
        """Small-strain 6x6 isotropic matrix (``neohookean.py:33-53``)."""
        lam = self._parameters.lame_parameter_1
        mu = self._parameters.shear_modulus
        C = np.zeros((6, 6), dtype=np.float64)
        C[0, 0] = C[1, 1] = C[2, 2] = lam + 2.0 * mu
        C[0, 1] = C[1, 0] = C[0, 2] = C[2, 0] = C[1, 2] = C[2, 1] = lam
        C[3, 3] = C[4, 4] = C[5, 5] = mu
        return C


class NeoHookeanField(NeoHookean):
    """NeoHookean with per-element shear and bulk moduli.

    ``mu_e``/``kappa_e`` are ``(E,)`` arrays (numpy or torch); ``lam_e`` defaults to
    ``kappa_e - 2/3 mu_e``.  ``parameters`` reports the first element's values so that
    code reading a scalar modulus still works.
    """

    def __init__(self, mu_e, kappa_e, mass_density: float = 1000.0, lam_e=None) -> None:
        self.mu_e = mu_e
        self.kappa_e = kappa_e
        self.lam_e = lam_e
        p = IsotropicElasticParameters()
        mu0 = float(np.asarray(_host(mu_e)).reshape(-1)[0])
        k0 = float(np.asarray(_host(kappa_e)).reshape(-1)[0])
        p.set_from_bulk_shear(bulk_modulus=k0, shear_modulus=mu0, mass_density=mass_density)
        super().__init__(p)


def _host(a):
    if hasattr(a, "detach"):
        return a.detach().cpu().numpy()
    return a


def material_moduli(material) -> tuple[float, float, float]:
    """(mu, kappa, lambda) of a reference or mirror material object."""
    p = material.parameters if hasattr(material, "parameters") else material._parameters
    return float(p.shear_modulus), float(p.bulk_modulus), float(p.lame_parameter_1)
