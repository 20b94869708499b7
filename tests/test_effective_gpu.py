"""Fused dynamic effective tangent c_t K_T + c_m M + c_0 K_0 (GPU).

The reference forms K_eff on the host from separately assembled matrices
(psierra analysis/nonlinear_dynamic.py:640-644); the fused sweep must equal that
combination: FP64 within 1e-13 of the largest entry, FP32-mixed within 2e-6.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import rel_max
from oracle.assembly import assemble_linear_stiffness, assemble_mass, assemble_tangent
from psierra_b200 import meshgen
from psierra_b200.assembler import GPUAssembler
from psierra_b200.material import IsotropicElasticParameters, NeoHookean, NeoHookeanField

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda")


def _nh(E=1e5, nu=0.35, rho=1040.0):
    p = IsotropicElasticParameters()
    p.set_from_youngs_poisson(youngs_modulus=E, poissons_ratio=nu, mass_density=rho)
    return NeoHookean(p)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-13), ("fp32-mixed", 2e-6)])
def test_fused_effective_tangent_equals_separate_assemblies(precision, tol):
    m = meshgen.box_tet4(1.0, 0.4, 0.3, 8, 4, 3)
    mat = _nh()
    asm = GPUAssembler(m.nodes, m.elements, mat, precision=precision)
    u = torch.from_numpy(meshgen.cantilever_seeded_u(m, seed=7).reshape(-1)).to(DEV)
    c_t, c_m, c_0 = 0.55, 3.7e4, 2.1e-3
    f_e, k_e = asm.assemble_effective(u, c_t, c_m, c_0)
    f1, k_t = asm.assemble(u, precision=precision)
    _, k_m = asm.assemble(None, mass=True, precision=precision)
    _, k_0 = asm.assemble(None, linear=True, precision=precision)
    ref = c_t * k_t.double() + c_m * k_m.double() + c_0 * k_0.double()
    assert rel_max(k_e.double().cpu().numpy(), ref.cpu().numpy()) < tol
    assert torch.equal(f_e, f1)
    # K-only request gives the same matrix
    _, k_only = asm.assemble_effective(u, c_t, c_m, c_0, want_f=False)
    assert torch.equal(k_only, k_e)


def test_effective_tangent_matches_oracle_and_per_element_moduli():
    m = meshgen.box_tet4(1.0, 0.3, 0.2, 5, 3, 2)
    rng = np.random.default_rng(4)
    mu = np.exp(np.log(2e4) + 0.3 * rng.normal(size=m.n_elements))
    kappa = 20.0 * mu
    field = NeoHookeanField(mu, kappa)
    asm = GPUAssembler(m.nodes, m.elements, field, precision="fp64")
    u_np = meshgen.cantilever_seeded_u(m, seed=3).reshape(-1)
    c_t, c_m, c_0, rho = 0.7, 1.3e3, 0.02, 900.0
    _, k_e = asm.assemble_effective(torch.from_numpy(u_np).to(DEV), c_t, c_m, c_0, rho=rho)
    Kt = assemble_tangent(m.nodes, m.elements, u_np.reshape(-1, 3), mu, kappa)
    Mo = assemble_mass(m.nodes, m.elements, rho)
    K0 = assemble_linear_stiffness(m.nodes, m.elements, kappa - 2.0 / 3.0 * mu, mu)
    ref = (c_t * Kt + c_m * Mo + c_0 * K0).tocsr()
    ref.sort_indices()
    assert np.array_equal(asm.pattern.indptr, ref.indptr) and np.array_equal(asm.pattern.indices, ref.indices)
    assert rel_max(k_e.cpu().numpy(), ref.data) < 1e-12
