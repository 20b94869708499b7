"""GPU parity of the Tet4 path against the reference's golden outputs and its test shapes.

Tolerances (FP64):
* K_T values: max |K - K_ref| / max |K_ref| <= 1e-13 (observed ~2e-14);
* f_int: ||f - f_ref||_2 / ||f_ref||_2 <= 1e-12.  The reference's own FP64 stress
  S = phi (I - I1/3 C^-1) + beta C^-1 cancels O(mu) terms at small strain, which
  puts ~1e-12 of rounding noise on its f_int; against an extended-precision
  evaluation the GPU kernel is accurate to ~1e-15.
FP32-mixed: K_T within 1e-6 (max-norm relative), f_int unchanged (FP64).
"""
from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse as spsp

from conftest import block_diagonal_blocks, disjoint_mesh, golden, rel_2, rel_max
from psierra_b200 import meshgen
from psierra_b200.element import Tet4TotalLagrangian
from psierra_b200.material import IsotropicElasticParameters, NeoHookean, NeoHookeanField

pytestmark = pytest.mark.gpu


def nh(E, nu, rho=1000.0):
    p = IsotropicElasticParameters()
    p.set_from_youngs_poisson(youngs_modulus=E, poissons_ratio=nu, mass_density=rho)
    return NeoHookean(p)


def nh_bulk_shear(kappa, mu):
    p = IsotropicElasticParameters()
    p.set_from_bulk_shear(bulk_modulus=kappa, shear_modulus=mu, mass_density=1000.0)
    return NeoHookean(p)


REGULAR_TET = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]])


@pytest.mark.parametrize("precision", ["fp64", "fp32-mixed"])
def test_random_elements_match_reference(precision):
    g = golden("element_tet4")
    n = len(g["X"])
    m = disjoint_mesh(g["X"])
    el = Tet4TotalLagrangian(NeoHookeanField(g["mu"], g["kappa"]), precision=precision)
    f, K = el.assemble_force_and_tangent(m, g["u"].reshape(-1, 3))
    kb = block_diagonal_blocks(K, n, 12)
    fb = f.reshape(n, 12)
    ktol = 1e-12 if precision == "fp64" else 1e-6
    for i in range(n):
        assert rel_max(kb[i], g["k"][i]) < ktol
        assert rel_max(fb[i], g["f"][i]) < 5e-12


def test_cfg1_seeded_state_fp64():
    g = golden("cfg1_seeded")
    m = meshgen.box_tet4(1.0, 0.1, 0.1, 40, 4, 4)
    el = Tet4TotalLagrangian(nh_bulk_shear(float(g["kappa"]), float(g["mu"])))
    f = el.assemble_internal_forces(m, g["u"])
    K = el.assemble_tangent_stiffness_matrix(m, g["u"])
    assert isinstance(K, spsp.csr_matrix) and K.has_sorted_indices
    assert np.array_equal(K.indptr, g["K_indptr"]) and np.array_equal(K.indices, g["K_indices"])
    assert rel_max(K.data, g["K_data"]) < 1e-13
    assert rel_2(f, g["f"]) < 1e-12
    # the fused sweep evaluates the same formulas; FMA contraction may differ by an ulp
    f2, K2 = el.assemble_force_and_tangent(m, g["u"])
    assert rel_max(f2, f) < 1e-14 and rel_max(K2.data, K.data) < 1e-14


def test_cfg1_fp32_mixed_error_bounds():
    g = golden("cfg1_seeded")
    m = meshgen.box_tet4(1.0, 0.1, 0.1, 40, 4, 4)
    el = Tet4TotalLagrangian(nh_bulk_shear(float(g["kappa"]), float(g["mu"])), precision="fp32-mixed")
    f, K = el.assemble_force_and_tangent(m, g["u"])
    assert rel_2(f, g["f"]) < 1e-12  # f_int stays FP64 in the mixed mode
    assert rel_max(K.data, g["K_data"]) < 1e-6
    assert rel_2(K.data, g["K_data"]) < 1e-6


def test_linear_stiffness_matches_reference():
    g = golden("cfg1_seeded")
    m = meshgen.box_tet4(1.0, 0.1, 0.1, 40, 4, 4)
    mat = nh(1e5, 0.3)
    assert abs(mat.parameters.lame_parameter_1 - float(g["lam"])) < 1e-9
    K = Tet4TotalLagrangian(mat).assemble_stiffness_matrix(m)
    assert rel_max(K.data, g["Klin_data"]) < 1e-13


def test_bitwise_reproducible():
    m = meshgen.box_tet4(1.0, 1.0, 1.0, 12, 12, 12)
    u = meshgen.cube_smooth_u(m, seed=5)
    for precision in ("fp64", "fp32-mixed"):
        el = Tet4TotalLagrangian(nh(3e3, 0.45), precision=precision)
        f0, K0 = el.assemble_force_and_tangent(m, u)
        for _ in range(10):
            f1, K1 = el.assemble_force_and_tangent(m, u)
            assert np.array_equal(f0, f1) and np.array_equal(K0.data, K1.data)


def test_rigid_translation_gives_zero_force():
    # reference tests/test_element_tet4_total_lagrangian.py:27-40
    el = Tet4TotalLagrangian(nh(200e9, 0.3, 7850.0))
    u = np.tile(np.array([12.5, -34.2, 5.8]), (4, 1))
    _, f = el.compute_nonlinear_force_and_tangent_stiffness(REGULAR_TET, u)
    assert np.allclose(f, 0.0, atol=1e-10)


def test_rigid_rotation_gives_zero_force():
    # reference tests/test_element_tet4_total_lagrangian.py:42-69
    el = Tet4TotalLagrangian(nh(10e3, 0.45))
    th = np.deg2rad(30.0)
    ax = np.ones(3) / np.sqrt(3.0)
    Km = np.array([[0, -ax[2], ax[1]], [ax[2], 0, -ax[0]], [-ax[1], ax[0], 0]])
    R = np.eye(3) + np.sin(th) * Km + (1.0 - np.cos(th)) * (Km @ Km)
    _, f = el.compute_nonlinear_force_and_tangent_stiffness(REGULAR_TET, REGULAR_TET @ R.T - REGULAR_TET)
    assert np.allclose(f, 0.0, atol=1e-10)


def test_small_strain_limit_matches_linear():
    # reference tests/test_element_tet4_total_lagrangian.py:71-91
    mat = nh(200e9, 0.3, 7850.0)
    el = Tet4TotalLagrangian(mat)
    K_lin = el.compute_linear_stiffness_matrix(REGULAR_TET)
    rng = np.random.RandomState(42)
    u = 1e-5 * rng.randn(4, 3)
    _, f = el.compute_nonlinear_force_and_tangent_stiffness(REGULAR_TET, u)
    fl = K_lin @ u.ravel()
    assert np.linalg.norm(f - fl) / np.linalg.norm(fl) < 1e-4


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-5), ("fp32-mixed", 1e-5)])
def test_tangent_matches_central_differences(precision, tol):
    # reference tests/test_element_tet4_total_lagrangian.py:93-132, on a 5-element patch
    m = meshgen.box_tet4(1.0, 1.0, 1.0, 1, 1, 1)
    rng = np.random.RandomState(123)
    u = 0.02 * rng.randn(m.n_nodes, 3)
    el = Tet4TotalLagrangian(nh(10e3, 0.45), precision=precision)
    K = el.assemble_tangent_stiffness_matrix(m, u).toarray()
    ref = Tet4TotalLagrangian(nh(10e3, 0.45))
    h = 1e-7
    Kfd = np.zeros_like(K)
    for d in range(m.n_dofs):
        up, um = u.copy().ravel(), u.copy().ravel()
        up[d] += h
        um[d] -= h
        Kfd[:, d] = (ref.assemble_internal_forces(m, up) - ref.assemble_internal_forces(m, um)) / (2 * h)
    assert np.linalg.norm(K - Kfd) / np.linalg.norm(K) < tol
    assert np.allclose(K, K.T, atol=1e-8 * np.abs(K).max())


@pytest.mark.parametrize("precision", ["fp64", "fp32-mixed"])  # fp32-mixed K: the warp-specialised kernel
def test_inverted_element_raises_reference_error(precision):
    m = meshgen.box_tet4(1.0, 1.0, 1.0, 2, 2, 2)
    u = np.zeros((m.n_nodes, 3))
    el = Tet4TotalLagrangian(nh(10e3, 0.45), precision=precision)
    f = el.assemble_internal_forces(m, u)
    assert np.abs(f).max() < 1e-12
    # push node 0 of element 7 through the opposite face
    e = 7
    c = m.nodes[m.elements[e]]
    centroid_opp = c[1:].mean(axis=0)
    u[m.elements[e, 0]] = 2.5 * (centroid_opp - c[0])
    def det_f(i):
        X = m.nodes[m.elements[i]]
        x = X + u[m.elements[i]]
        return np.linalg.det(x[1:] - x[0]) / np.linalg.det(X[1:] - X[0])

    bad = [i for i in range(m.n_elements) if det_f(i) <= 0]
    assert bad and min(bad) <= e
    Jref = det_f(min(bad))
    with pytest.raises(ValueError, match="Element inversion detected") as ei:
        el.assemble_internal_forces(m, u)
    assert f"{Jref:.4e}" in str(ei.value)
    with pytest.raises(ValueError, match="Element inversion detected") as ei:
        el.assemble_tangent_stiffness_matrix(m, u)
    assert f"{Jref:.4e}" in str(ei.value)
    with pytest.raises(ValueError, match="Element inversion detected"):
        el.assemble_force_and_tangent(m, u)


def test_negative_volume_raises_reference_error():
    m = meshgen.box_tet4(1.0, 1.0, 1.0, 1, 1, 1)
    els = m.elements.copy()
    els[3, [1, 2]] = els[3, [2, 1]]
    bad = meshgen.TetMesh(m.nodes, els)
    el = Tet4TotalLagrangian(nh(10e3, 0.45))
    with pytest.raises(ValueError, match="Negative or zero element volume detected"):
        el.assemble_internal_forces(bad, np.zeros((m.n_nodes, 3)))


@pytest.mark.parametrize("precision", ["fp64", "fp32-mixed"])
def test_per_element_api_reuses_one_assembler(precision):
    """compute_nonlinear_force_and_tangent_stiffness / compute_linear_stiffness_matrix called
    element by element on one object (as reference loops over elements do): the cached
    one-element assembler is built once and gives each golden element's k, f and k_lin."""
    g = golden("element_tet4")
    el = Tet4TotalLagrangian(NeoHookeanField(g["mu"], g["kappa"], lam_e=g["lam"]), precision=precision)
    ktol = 1e-12 if precision == "fp64" else 1e-6
    first = None
    for i in range(16):
        k, f = el.compute_nonlinear_force_and_tangent_stiffness(g["X"][i], g["u"][i], elem_index=i)
        assert rel_max(k, g["k"][i]) < ktol and rel_max(f, g["f"][i]) < 5e-12
        kl = el.compute_linear_stiffness_matrix(g["X"][i], elem_index=i)
        assert rel_max(kl, g["k_lin"][i]) < ktol
        one = el._one[0]._asm
        first = first or one
        assert one is first  # built once
