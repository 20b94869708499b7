"""Tet4Fbar on the GPU against the reference (golden fixture) and the oracle.

Tolerances: FP64 path, 1e-12 relative to the largest entry (the oracle itself matches the
reference to that bound).  The tangent's CSR pattern must be the reference's.
"""
from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse as spsp

from conftest import golden
from oracle import tet4fbar
from psierra_b200 import meshgen
from psierra_b200.element import Tet4Fbar
from psierra_b200.material import IsotropicElasticParameters, NeoHookean

pytestmark = pytest.mark.gpu


def _nh(E, nu):
    p = IsotropicElasticParameters()
    p.set_from_youngs_poisson(youngs_modulus=E, poissons_ratio=nu, mass_density=1000.0)
    return NeoHookean(p)


def _rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max()


def test_fbar_matches_reference_fixture():
    g = golden("fbar_box")
    m = meshgen.TetMesh(g["nodes"], g["elements"])
    el = Tet4Fbar(_nh(1e4, 0.45))
    f = el.assemble_internal_forces(m, g["u"])
    assert _rel(f, g["f"]) < 1e-12
    assert np.abs(el._domain_J_bar - g["J_bar"]).max() < 1e-14
    K = el.assemble_tangent_stiffness_matrix(m, g["u"])
    Kr = spsp.csr_matrix((g["K_data"], g["K_indices"], g["K_indptr"]), shape=K.shape)
    assert np.array_equal(K.indptr, Kr.indptr) and np.array_equal(K.indices, Kr.indices)
    assert _rel(K.data, Kr.data) < 1e-12
    # at u = 0 (F = I) entries that vanish exactly come out as rounding noise in the
    # reference's dense products (and so stay in its pattern) but as exact zeros in the
    # closed form: the values agree on the union of the patterns, and an entry present in
    # only one of them is below the noise level
    K0 = el.assemble_stiffness_matrix(m)
    K0r = spsp.csr_matrix((g["Klin_data"], g["Klin_indices"], g["Klin_indptr"]), shape=K.shape)
    scale = np.abs(K0r.data).max()
    assert np.abs((K0 - K0r).toarray()).max() <= 1e-12 * scale
    ours = set(zip(*K0.nonzero()))
    ref = K0r.tocoo()
    for r, c, v in zip(ref.row, ref.col, ref.data):
        if (r, c) not in ours:
            assert abs(v) <= 1e-13 * scale
    for i, e in enumerate(g["pick"]):
        k, fe = el.compute_nonlinear_force_and_tangent_stiffness(g["nodes"][g["elements"][e]], g["u"][g["elements"][e]],
                                                                 J_bar=float(g["pick_J_bar"][i]))
        assert _rel(k, g["pick_k"][i]) < 1e-12 and _rel(fe, g["pick_f"][i]) < 1e-12


def test_fbar_matches_oracle_on_a_larger_deformed_mesh():
    m = meshgen.box_tet4(1.0, 0.6, 0.5, 7, 4, 3)
    u = meshgen.cantilever_seeded_u(m, seed=17) * 20.0
    mat = _nh(2e4, 0.49)
    mu, kappa = mat.parameters.shear_modulus, mat.parameters.bulk_modulus
    el = Tet4Fbar(mat)
    f, K = el.assemble_force_and_tangent(m, u)
    fo = tet4fbar.internal_forces(m.nodes, m.elements, u, mu, kappa)
    Ko = tet4fbar.tangent(m.nodes, m.elements, u, mu, kappa)
    assert _rel(f, fo) < 1e-12
    assert np.abs((K - Ko).toarray()).max() <= 1e-12 * np.abs(Ko.data).max()
    assert abs(K - K.T).max() <= 1e-12 * np.abs(K.data).max()
    # reproducible to the bit
    f2, K2 = el.assemble_force_and_tangent(m, u)
    assert np.array_equal(f, f2) and np.array_equal(K.data, K2.data)


def test_fbar_inversion_error_names_the_element():
    m = meshgen.box_tet4(1.0, 0.3, 0.3, 3, 1, 1)
    u = np.zeros((m.n_nodes, 3))
    tip = meshgen.nodes_on_plane(m, 0, "max")
    u[tip, 0] = -1.5  # pushes the last cells through themselves
    el = Tet4Fbar(_nh(1e4, 0.3))
    with pytest.raises(ValueError, match=r"Element inversion detected at element \d+: det\(F\) = .* <= 0\."):
        el.assemble_internal_forces(m, u)
