"""Hyper-reduced (ECSW) evaluation against the reference formula (GPU).

f_r = sum_e w_e Phi_e^T f_e, K_r = sym(sum_e w_e Phi_e^T k_e Phi_e) with the per-element
(k, f) of the oracle (hyperreduction/model.py:254-318); FP64, 1e-12 relative.
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle.tet4 import force_and_tangent
from psierra_b200 import meshgen
from psierra_b200.ecsw import ECSWEvaluator
from psierra_b200.material import IsotropicElasticParameters, NeoHookean, NeoHookeanField

pytestmark = pytest.mark.gpu


def _reference(m, Phi, idx, w, u_r, mu, kappa):
    r = Phi.shape[1]
    f_r = np.zeros(r)
    K_r = np.zeros((r, r))
    for e, we in zip(idx, w):
        nodes = m.elements[e]
        dofs = (3 * nodes[:, None] + np.arange(3)).ravel()
        Pe = Phi[dofs]
        ue = (Pe @ u_r).reshape(4, 3)
        mue = mu[e] if np.ndim(mu) else mu
        kae = kappa[e] if np.ndim(kappa) else kappa
        k, f = force_and_tangent(m.nodes[nodes], ue, mue, kae)
        f_r += we * (Pe.T @ f)
        K_r += we * (Pe.T @ (k @ Pe))
    return f_r, 0.5 * (K_r + K_r.T)


@pytest.mark.parametrize("per_element", [False, True])
def test_ecsw_matches_reference_formula(per_element):
    m = meshgen.box_tet4(1.0, 0.4, 0.3, 6, 3, 2)
    rng = np.random.default_rng(8)
    r = 10
    Phi, _ = np.linalg.qr(rng.normal(size=(m.n_dofs, r)))
    idx = np.sort(rng.choice(m.n_elements, size=40, replace=False))
    w = rng.uniform(0.5, 3.0, size=idx.size)
    u_r = 0.05 * rng.normal(size=r)
    p = IsotropicElasticParameters()
    p.set_from_youngs_poisson(youngs_modulus=1e4, poissons_ratio=0.4, mass_density=1000.0)
    if per_element:
        mu = p.shear_modulus * np.exp(0.2 * rng.normal(size=m.n_elements))
        kappa = 30.0 * mu
        mat = NeoHookeanField(mu, kappa)
    else:
        mat = NeoHookean(p)
        mu, kappa = p.shear_modulus, p.bulk_modulus
    ev = ECSWEvaluator(m.nodes, m.elements, mat, Phi, idx, w)
    f, K = ev.evaluate_forces_and_stiffness(u_r)
    fr, Kr = _reference(m, Phi, idx, w, u_r, mu, kappa)
    assert np.abs(f - fr).max() <= 1e-12 * np.abs(fr).max()
    assert np.abs(K - Kr).max() <= 1e-12 * np.abs(Kr).max()
    assert np.array_equal(K, K.T)
    f2, K2 = ev.evaluate_forces_and_stiffness(u_r)
    assert np.array_equal(f, f2) and np.array_equal(K, K2)
