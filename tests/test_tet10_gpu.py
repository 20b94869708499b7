"""GPU parity of the Tet10 path against the reference's golden outputs and its test shapes
(psierra tests/test_element_tet10_total_lagrangian.py)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import block_diagonal_blocks, disjoint_mesh, golden, rel_2, rel_max
from oracle import vectorized
from psierra_b200 import meshgen
from psierra_b200.element import Tet10TotalLagrangian
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


def tet10_coords():
    v = np.array([[0.0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]])
    e = [(0, 1), (1, 2), (2, 0), (0, 3), (1, 3), (2, 3)]
    return np.vstack([v] + [0.5 * (v[a] + v[b])[None] for a, b in e])


@pytest.mark.parametrize("precision", ["fp64", "fp32-mixed"])
def test_random_tet10_elements_match_reference(precision):
    g = golden("element_tet10")
    n = len(g["X"])
    m = disjoint_mesh(g["X"])
    el = Tet10TotalLagrangian(NeoHookeanField(g["mu"], g["kappa"]), precision=precision)
    f, K = el.assemble_force_and_tangent(m, g["u"].reshape(-1, 3))
    kb = block_diagonal_blocks(K, n, 30)
    fb = f.reshape(n, 30)
    ktol = 1e-12 if precision == "fp64" else 2e-6
    for i in range(n):
        assert rel_max(kb[i], g["k"][i]) < ktol
        assert rel_max(fb[i], g["f"][i]) < 5e-12


def test_tet10_box_matches_reference():
    g = golden("tet10_box3")
    m = meshgen.TetMesh(g["nodes"], g["elements"])
    el = Tet10TotalLagrangian(nh_bulk_shear(float(g["kappa"]), float(g["mu"])))
    f, K = el.assemble_force_and_tangent(m, g["u"])
    assert np.array_equal(K.indptr, g["K_indptr"]) and np.array_equal(K.indices, g["K_indices"])
    assert rel_max(K.data, g["K_data"]) < 1e-13
    assert rel_2(f, g["f"]) < 1e-12
    f1 = el.assemble_internal_forces(m, g["u"])
    assert rel_2(f1, g["f"]) < 1e-12
    mat = nh_bulk_shear(float(g["kappa"]), float(g["mu"]))
    Kl = Tet10TotalLagrangian(mat).assemble_stiffness_matrix(m)
    assert rel_max(Kl.data, g["Klin_data"]) < 1e-13


def test_tet10_larger_mesh_against_oracle_and_reproducible():
    m = meshgen.tet4_to_tet10(meshgen.box_tet4(1.0, 1.0, 1.0, 6, 5, 7))
    u = meshgen.cube_smooth_u(m, seed=3)
    mat = nh(1e4, 0.4)
    fo, Ko = vectorized.assemble_force_and_tangent(m.nodes, m.elements, u, mat.parameters.shear_modulus,
                                                   mat.parameters.bulk_modulus)
    for precision, tol in (("fp64", 1e-12), ("fp32-mixed", 2e-6)):
        el = Tet10TotalLagrangian(mat, precision=precision)
        f, K = el.assemble_force_and_tangent(m, u)
        assert np.array_equal(K.indptr, Ko.indptr) and np.array_equal(K.indices, Ko.indices)
        assert rel_max(K.data, Ko.data) < tol
        assert rel_2(f, fo) < 1e-11
        f2, K2 = el.assemble_force_and_tangent(m, u)
        assert np.array_equal(f, f2) and np.array_equal(K.data, K2.data)


def test_tet10_translation_and_rotation():
    X = tet10_coords()
    el = Tet10TotalLagrangian(nh(10e3, 0.45))
    _, f = el.compute_nonlinear_force_and_tangent_stiffness(X, np.tile([3.0, -2.0, 7.5], (10, 1)))
    assert np.allclose(f, 0.0, atol=1e-10)
    th = np.deg2rad(25.0)
    R = np.array([[np.cos(th), -np.sin(th), 0], [np.sin(th), np.cos(th), 0], [0, 0, 1.0]])
    _, f = el.compute_nonlinear_force_and_tangent_stiffness(X, X @ R.T - X)
    assert np.allclose(f, 0.0, atol=1e-7)


def test_tet10_tangent_matches_central_differences():
    # reference tests/test_element_tet10_total_lagrangian.py:136-176 on a 2-element patch
    m = meshgen.tet4_to_tet10(meshgen.TetMesh(np.array([[0.0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 1.0]]),
                                              np.array([[0, 1, 2, 3], [1, 2, 3, 4]])))
    rng = np.random.RandomState(42)
    u = 0.01 * rng.randn(m.n_nodes, 3)
    el = Tet10TotalLagrangian(nh(10e3, 0.45))
    K = el.assemble_tangent_stiffness_matrix(m, u).toarray()
    h = 1e-7
    Kfd = np.zeros_like(K)
    for d in range(m.n_dofs):
        up, um = u.copy().ravel(), u.copy().ravel()
        up[d] += h
        um[d] -= h
        Kfd[:, d] = (el.assemble_internal_forces(m, up) - el.assemble_internal_forces(m, um)) / (2 * h)
    assert np.linalg.norm(K - Kfd) / np.linalg.norm(K) < 1e-5
    assert np.allclose(K, K.T, atol=1e-8 * np.abs(K).max())


def test_tet10_inversion_error():
    X = tet10_coords()
    u = np.zeros((10, 3))
    u[3] = [0.0, 0.0, -2.0]  # corner 3 through the opposite face
    with pytest.raises(ValueError, match="Element inversion detected|Negative or zero Jacobian"):
        Tet10TotalLagrangian(nh(10e3, 0.45)).compute_nonlinear_force_and_tangent_stiffness(X, u)


def test_tet10_prescribed_compression_matches_reference_newton():
    """The Tet10 cube solve at a reduced grid through the device Newton (GPU assembly,
    symmetric elimination, block-Jacobi PCG) against the reference's Newton with its
    direct solver: same iteration counts, displacement within 1e-8."""
    import torch

    from psierra_b200.assembler import GPUAssembler
    from psierra_b200.newton import DeviceNewton

    g = golden("tet10_newton")
    m = meshgen.tet4_to_tet10(meshgen.box_tet4(1.0, 1.0, 1.0, 3, 3, 3))
    E = m.n_elements
    asm = GPUAssembler(m.nodes, m.elements, NeoHookeanField(np.full(E, float(g["mu"])), np.full(E, float(g["kappa"]))))
    bottom, top = g["bottom"], g["top"]
    fixed = np.concatenate([3 * bottom + c for c in range(3)] + [3 * top + 2])
    up = np.zeros(m.n_dofs)
    up[3 * top + 2] = -0.2
    nt = DeviceNewton(asm, fixed, precision="fp64", pcg_tol=1e-13)
    res = nt.solve(torch.zeros(m.n_dofs, dtype=torch.float64, device="cuda"),
                   u_prescribed=torch.from_numpy(up).cuda(), n_steps=8, nr_iterations=20, nr_tol=1e-8)
    assert res.converged and bool(g["converged"])
    assert res.iteration_history == g["iterations"].tolist()
    assert np.abs(res.u.cpu().numpy() - g["u"]).max() <= 1e-8 * np.abs(g["u"]).max()


@pytest.mark.parametrize("precision", ["fp64", "fp32-mixed"])
def test_tet10_compression_workload_loading_matches_reference_newton(precision):
    """The Tet10 compression workload's loading (top face u_z = -0.2 over 20 increments,
    Jacobi PCG, Newton tolerance 1e-8) on 6^3 cells -> 1,296 Tet10 through the device
    Newton, against the reference's Newton with its direct solver
    (analysis/nonlinear_static.py:250-404).  FP64: the same iteration counts and the
    displacement within 1e-10; FP32-mixed tangent (the residual stays FP64, so Newton
    still converges to the FP64 equilibrium): within 1e-8."""
    import torch

    from psierra_b200.assembler import GPUAssembler
    from psierra_b200.newton import DeviceNewton

    g = golden("tet10_compress6")
    cells, n_steps = int(g["cells"]), int(g["n_steps"])
    m = meshgen.tet4_to_tet10(meshgen.box_tet4(1.0, 1.0, 1.0, cells, cells, cells))
    E = m.n_elements
    asm = GPUAssembler(m.nodes, m.elements, NeoHookeanField(np.full(E, float(g["mu"])), np.full(E, float(g["kappa"]))))
    bottom, top = g["bottom"], g["top"]
    fixed = np.concatenate([3 * bottom + c for c in range(3)] + [3 * top + 2])
    up = np.zeros(m.n_dofs)
    up[3 * top + 2] = -0.2
    nt = DeviceNewton(asm, fixed, precision=precision, pcg_tol=1e-13, pcg_maxiter=100000, preconditioner="jacobi")
    res = nt.solve(torch.zeros(m.n_dofs, dtype=torch.float64, device="cuda"),
                   u_prescribed=torch.from_numpy(up).cuda(), n_steps=n_steps, nr_iterations=30, nr_tol=1e-8)
    assert res.converged and bool(g["converged"])
    if precision == "fp64":
        assert res.iteration_history == g["iterations"].tolist()
    tol = 1e-10 if precision == "fp64" else 1e-8
    assert np.abs(res.u.cpu().numpy() - g["u"]).max() <= tol * np.abs(g["u"]).max()
