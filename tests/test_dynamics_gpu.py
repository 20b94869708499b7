"""Device generalized-alpha dynamics against the reference NonlinearDynamicAnalysis (GPU)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import golden, rel_2
from psierra_b200 import meshgen
from psierra_b200.assembler import GPUAssembler
from psierra_b200.dynamics import DeviceGeneralizedAlpha
from psierra_b200.material import IsotropicElasticParameters, NeoHookean

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda")


def _beam(g):
    m = meshgen.box_tet4(1.0, 0.1, 0.1, 8, 2, 2)
    p = IsotropicElasticParameters()
    p.set_from_youngs_poisson(youngs_modulus=1e5, poissons_ratio=0.3, mass_density=float(g["rho"]))
    return m, NeoHookean(p)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-8), ("fp32-mixed", 1e-6)])
def test_generalized_alpha_matches_reference_trajectory(precision, tol):
    g = golden("dynamic_beam")
    m, mat = _beam(g)
    asm = GPUAssembler(m.nodes, m.elements, mat, precision=precision)
    fixed = np.concatenate([3 * g["clamp"] + c for c in range(3)])
    dyn = DeviceGeneralizedAlpha(asm, fixed, damping=tuple(g["rayleigh"]), spectral_radius=float(g["spectral_radius"]),
                                 pcg_tol=1e-13)
    res = dyn.solve(torch.from_numpy(g["f_ext"]).to(DEV), dt=float(g["dt"]), n_steps=int(g["n_steps"]),
                    nr_iterations=15, nr_tol=float(g["nr_tol"]))
    assert res.converged and bool(g["converged"])
    if precision == "fp64":
        assert res.iteration_history == g["iterations"].tolist()
    assert rel_2(res.u.cpu().numpy(), g["u"]) < tol
    assert rel_2(res.v.cpu().numpy(), g["v"]) < 10 * tol
    assert rel_2(res.a.cpu().numpy(), g["a"]) < 100 * tol


def test_effective_tangent_constants_match_separate_assembly():
    """The driver's fused K_eff equals (1-af) K_T + (1-am) a0 M + (1-af) a1 (aR M + bR K0)."""
    g = golden("dynamic_beam")
    m, mat = _beam(g)
    asm = GPUAssembler(m.nodes, m.elements, mat, precision="fp64")
    fixed = np.concatenate([3 * g["clamp"] + c for c in range(3)])
    dyn = DeviceGeneralizedAlpha(asm, fixed, damping=(0.5, 1e-4), spectral_radius=0.8)
    dt = 0.05
    am, af, ga, be = dyn.alpha_m, dyn.alpha_f, dyn.gamma, dyn.beta
    assert abs(am - (2 * 0.8 - 1) / 1.8) < 1e-15 and abs(af - 0.8 / 1.8) < 1e-15
    a0, a1 = 1.0 / (be * dt ** 2), ga / (be * dt)
    u = torch.from_numpy(meshgen.cantilever_seeded_u(m, seed=5).reshape(-1)).to(DEV)
    _, ke = asm.assemble_effective(u, 1 - af, (1 - am) * a0 + (1 - af) * a1 * 0.5, (1 - af) * a1 * 1e-4)
    _, kt = asm.assemble(u)
    want = (1 - af) * kt + ((1 - am) * a0 + (1 - af) * a1 * 0.5) * dyn.M + (1 - af) * a1 * 1e-4 * dyn.K0
    assert (ke - want).abs().max().item() <= 1e-13 * want.abs().max().item()


def _beam10():
    g = golden("dynamic_tet10")
    m = meshgen.tet4_to_tet10(meshgen.box_tet4(1.0, 0.1, 0.1, 6, 2, 2))
    p = IsotropicElasticParameters()
    p.set_from_youngs_poisson(youngs_modulus=1e5, poissons_ratio=0.3, mass_density=float(g["rho"]))
    return g, m, NeoHookean(p)


def test_tet10_consistent_mass_matches_reference():
    """The device Tet10 mass (psx_tet10_assemble with PSX_MASS) against the reference domain's
    assemble_mass_matrix (element/tet10_base.py:344-372): same CSR, values within 1e-14."""
    g, m, mat = _beam10()
    for precision, tol in (("fp64", 1e-14), ("fp32-mixed", 1e-7)):
        asm = GPUAssembler(m.nodes, m.elements, mat, precision=precision)
        _, mv = asm.assemble(None, mass=True)
        assert np.array_equal(asm.pattern.indptr, g["M_indptr"]) and np.array_equal(asm.pattern.indices,
                                                                                       g["M_indices"])
        ref = g["M_data"]
        assert np.abs(mv.double().cpu().numpy() - ref).max() <= tol * np.abs(ref).max()


def test_tet10_effective_tangent_matches_separate_assembly():
    g, m, mat = _beam10()
    asm = GPUAssembler(m.nodes, m.elements, mat, precision="fp64")
    u = torch.from_numpy(meshgen.cantilever_seeded_u(m, seed=3).reshape(-1)).to(DEV)
    c_t, c_m, c_0 = 0.55, 812.5, 0.031
    f, ke = asm.assemble_effective(u, c_t, c_m, c_0)
    f2, kt = asm.assemble(u)
    _, M = asm.assemble(None, mass=True)
    _, K0 = asm.assemble(None, linear=True)
    want = c_t * kt + c_m * M + c_0 * K0
    assert torch.equal(f, f2)
    assert (ke - want).abs().max().item() <= 1e-14 * want.abs().max().item()


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-8), ("fp32-mixed", 1e-6)])
def test_tet10_generalized_alpha_matches_reference_trajectory(precision, tol):
    g, m, mat = _beam10()
    asm = GPUAssembler(m.nodes, m.elements, mat, precision=precision)
    fixed = np.concatenate([3 * g["clamp"] + c for c in range(3)])
    dyn = DeviceGeneralizedAlpha(asm, fixed, damping=tuple(g["rayleigh"]), spectral_radius=float(g["spectral_radius"]),
                                 pcg_tol=1e-13)
    res = dyn.solve(torch.from_numpy(g["f_ext"]).to(DEV), dt=float(g["dt"]), n_steps=int(g["n_steps"]),
                    nr_iterations=15, nr_tol=float(g["nr_tol"]))
    assert res.converged and bool(g["converged"])
    if precision == "fp64":
        assert res.iteration_history == g["iterations"].tolist()
    assert rel_2(res.u.cpu().numpy(), g["u"]) < tol
    assert rel_2(res.v.cpu().numpy(), g["v"]) < 10 * tol
    assert rel_2(res.a.cpu().numpy(), g["a"]) < 100 * tol
