"""The CPU oracle (numpy restatement of the reference) against the reference's own outputs.

The golden vectors were produced by running pSierra itself
(``tests/golden/make_golden.py``); these tests pin the oracle before any GPU result
is compared with it.
"""
from __future__ import annotations

import numpy as np

from conftest import golden, rel_max
from oracle import assembly, neohookean, tet4, tet10, vectorized
from psierra_b200 import meshgen


def test_neohookean_matches_reference():
    g = golden("material_nh")
    for F, C, S in zip(g["F"], g["C"], g["S"]):
        Co, So = neohookean.stress_and_tangent(F, float(g["mu"]), float(g["kappa"]))
        assert np.array_equal(Co, C) or rel_max(Co, C) < 1e-14
        assert np.array_equal(So, S) or rel_max(So, S) < 1e-14


def test_tet4_elements_match_reference():
    g = golden("element_tet4")
    for i in range(len(g["X"])):
        k, f = tet4.force_and_tangent(g["X"][i], g["u"][i], g["mu"][i], g["kappa"][i])
        assert rel_max(k, g["k"][i]) < 1e-14
        assert rel_max(f, g["f"][i]) < 1e-14
        kl = tet4.linear_stiffness(g["X"][i], g["lam"][i], g["mu"][i])
        assert rel_max(kl, g["k_lin"][i]) < 1e-14


def test_tet10_elements_match_reference():
    g = golden("element_tet10")
    for i in range(len(g["X"])):
        k, f = tet10.force_and_tangent(g["X"][i], g["u"][i], g["mu"][i], g["kappa"][i])
        assert rel_max(k, g["k"][i]) < 1e-14
        assert rel_max(f, g["f"][i]) < 1e-14
        kl = tet10.linear_stiffness(g["X"][i], g["lam"][i], g["mu"][i])
        assert rel_max(kl, g["k_lin"][i]) < 1e-14


def test_vectorized_matches_reference_elements():
    for name, npe in (("element_tet4", 4), ("element_tet10", 10)):
        g = golden(name)
        n = len(g["X"])
        nodes = g["X"].reshape(-1, 3)
        els = np.arange(n * npe).reshape(n, npe)
        k, f = vectorized.element_force_and_tangent(nodes, els, g["u"].reshape(-1, 3), g["mu"], g["kappa"])
        for i in range(n):
            # elementwise cancellation in the reference's S formula bounds the f agreement
            assert rel_max(k[i], g["k"][i]) < 1e-12
            assert rel_max(f[i], g["f"][i]) < 5e-12


def test_oracle_matches_reference_at_extreme_states():
    """Large stretch and compression with rotation (det F 0.35 to 2.5), Poisson ratios up
    to 0.4999, and strains of 1e-7 (every fourth element), from the reference's element."""
    for name, npe, mod in (("element_extreme_tet4", 4, tet4), ("element_extreme_tet10", 10, tet10)):
        g = golden(name)
        n = len(g["X"])
        assert {0.35, 0.6, 1.8, 2.5} <= set(np.round(g["det_F"], 6)) and max(g["nu"]) == 0.4999
        for i in range(n):
            k, f = mod.force_and_tangent(g["X"][i], g["u"][i], g["mu"][i], g["kappa"][i])
            assert rel_max(k, g["k"][i]) < 1e-15 and rel_max(f, g["f"][i]) < 1e-15  # step for step
        nodes = g["X"].reshape(-1, 3)
        els = np.arange(n * npe).reshape(n, npe)
        k, f = vectorized.element_force_and_tangent(nodes, els, g["u"].reshape(-1, 3), g["mu"], g["kappa"])
        for i in range(n):
            assert rel_max(k[i], g["k"][i]) < 5e-13
            if i % 4 == 3:
                # strain 1e-7: the reference's S = phi (I - I1/3 C^-1) + beta C^-1 makes f
                # accurate to about 1e-16 / 1e-7 = 1e-9 relative, so another association
                # agrees to ~1e-8 only
                assert rel_max(f[i], g["f"][i]) < 2e-7
            else:
                assert rel_max(f[i], g["f"][i]) < 1e-12


def test_cfg1_assembly_matches_reference():
    g = golden("cfg1_seeded")
    m = meshgen.box_tet4(1.0, 0.1, 0.1, 40, 4, 4)
    assert np.array_equal(meshgen.cantilever_seeded_u(m, seed=int(g["seed"])), g["u"])
    f, K = assembly.assemble_force_and_tangent(m.nodes, m.elements, g["u"], float(g["mu"]), float(g["kappa"]))
    assert np.array_equal(K.indptr, g["K_indptr"]) and np.array_equal(K.indices, g["K_indices"])
    assert rel_max(K.data, g["K_data"]) < 1e-15
    assert rel_max(f, g["f"]) < 1e-15
    Kl = assembly.assemble_linear_stiffness(m.nodes, m.elements, float(g["lam"]), float(g["mu"]))
    assert rel_max(Kl.data, g["Klin_data"]) < 1e-15


def test_tet10_box_matches_reference():
    g = golden("tet10_box3")
    m = meshgen.tet4_to_tet10(meshgen.box_tet4(1.0, 1.0, 1.0, 3, 3, 3))
    assert np.array_equal(m.elements, g["elements"]) and np.array_equal(m.nodes, g["nodes"])
    f, K = vectorized.assemble_force_and_tangent(m.nodes, m.elements, g["u"], float(g["mu"]), float(g["kappa"]))
    assert np.array_equal(K.indptr, g["K_indptr"]) and np.array_equal(K.indices, g["K_indices"])
    assert rel_max(K.data, g["K_data"]) < 1e-13
    assert rel_max(f, g["f"]) < 1e-11


def test_fbar_oracle_matches_reference_fixture():
    """oracle/tet4fbar.py against the reference Tet4Fbar run through SolidDomain."""
    import scipy.sparse as spsp

    from oracle import tet4fbar

    g = golden("fbar_box")
    nodes, el, u = g["nodes"], g["elements"], g["u"]
    mu, kappa = float(g["mu"]), float(g["kappa"])
    f = tet4fbar.internal_forces(nodes, el, u, mu, kappa)
    assert np.abs(f - g["f"]).max() <= 1e-12 * np.abs(g["f"]).max()
    K = tet4fbar.tangent(nodes, el, u, mu, kappa)
    Kr = spsp.csr_matrix((g["K_data"], g["K_indices"], g["K_indptr"]), shape=K.shape)
    assert np.abs((K - Kr).toarray()).max() <= 1e-12 * np.abs(Kr.data).max()
    assert K.nnz == Kr.nnz and np.array_equal(K.indptr, Kr.indptr) and np.array_equal(K.indices, Kr.indices)
    K0 = tet4fbar.tangent(nodes, el, np.zeros_like(u), mu, kappa)
    K0r = spsp.csr_matrix((g["Klin_data"], g["Klin_indices"], g["Klin_indptr"]), shape=K.shape)
    assert np.abs((K0 - K0r).toarray()).max() <= 1e-12 * np.abs(K0r.data).max()
    H, V, v0 = tet4fbar.geometry(nodes, el)
    _, J = tet4fbar.jacobians(el, u, H)
    _, Jb = tet4fbar.j_bar(el, V, J, v0)
    assert np.abs(Jb - g["J_bar"]).max() <= 1e-14
    for i, e in enumerate(g["pick"]):
        k, fe = tet4fbar.element_force_and_tangent(nodes[el[e]], u[el[e]], mu, kappa, float(g["pick_J_bar"][i]))
        assert np.abs(k - g["pick_k"][i]).max() <= 1e-12 * np.abs(g["pick_k"][i]).max()
        assert np.abs(fe - g["pick_f"][i]).max() <= 1e-12 * np.abs(g["pick_f"][i]).max()
