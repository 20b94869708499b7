"""Matrix-free K_T(u) v and the fused dynamic-relaxation step against the assembled tangent.

The oracle is the reference's assembled K_T (golden cfg1 values, and the assembled
CSR of this library for larger meshes) times v in FP64 on the host.
"""
from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse as spsp
import torch

from conftest import golden, rel_2
from psierra_b200 import meshgen
from psierra_b200.assembler import GPUAssembler
from psierra_b200.material import IsotropicElasticParameters, NeoHookean

pytestmark = pytest.mark.gpu


def nh(E, nu):
    p = IsotropicElasticParameters()
    p.set_from_youngs_poisson(youngs_modulus=E, poissons_ratio=nu, mass_density=1000.0)
    return NeoHookean(p)


def nh_bulk_shear(kappa, mu):
    p = IsotropicElasticParameters()
    p.set_from_bulk_shear(bulk_modulus=kappa, shear_modulus=mu, mass_density=1000.0)
    return NeoHookean(p)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-13), ("fp32-mixed", 2e-6)])
def test_kv_matches_reference_tangent_product(precision, tol):
    g = golden("cfg1_seeded")
    m = meshgen.box_tet4(1.0, 0.1, 0.1, 40, 4, 4)
    K = spsp.csr_matrix((g["K_data"], g["K_indices"], g["K_indptr"]), shape=(m.n_dofs, m.n_dofs))
    asm = GPUAssembler(m.nodes, m.elements, nh_bulk_shear(float(g["kappa"]), float(g["mu"])), precision=precision)
    rng = np.random.default_rng(0)
    v = rng.normal(size=m.n_dofs)
    u_d = torch.from_numpy(g["u"].reshape(-1)).cuda()
    y = asm.kv(u_d, torch.from_numpy(v).cuda()).cpu().numpy()
    assert rel_2(y, K @ v) < tol


def test_kv_matches_assembled_csr_and_is_reproducible():
    m = meshgen.box_tet4(1.0, 1.0, 1.0, 16, 14, 12)
    u = meshgen.cube_smooth_u(m, seed=9)
    asm = GPUAssembler(m.nodes, m.elements, nh(3e3, 0.45))
    u_d = torch.from_numpy(u.reshape(-1)).cuda()
    _, k = asm.assemble(u_d, want_f=False, want_k=True)
    p = asm.pattern
    K = spsp.csr_matrix((k.cpu().numpy(), p.indices, p.indptr), shape=(p.n_dofs, p.n_dofs))
    v = torch.randn(p.n_dofs, dtype=torch.float64, device="cuda")
    y1 = asm.kv(u_d, v).cpu().numpy()
    y2 = asm.kv(u_d, v).cpu().numpy()
    assert np.array_equal(y1, y2)
    assert rel_2(y1, K @ v.cpu().numpy()) < 1e-13


def test_fused_dr_steps_match_host_iteration():
    m = meshgen.box_tet4(1.0, 0.2, 0.2, 12, 3, 3)
    u = meshgen.cantilever_seeded_u(m, seed=4)
    asm = GPUAssembler(m.nodes, m.elements, nh(1e5, 0.3))
    u_d = torch.from_numpy(u.reshape(-1)).cuda()
    _, k = asm.assemble(u_d, want_f=False, want_k=True)
    p = asm.pattern
    K = spsp.csr_matrix((k.cpu().numpy(), p.indices, p.indptr), shape=(p.n_dofs, p.n_dofs))
    n = p.n_dofs
    rng = np.random.default_rng(1)
    b = rng.normal(size=n)
    # Gerschgorin mass of analysis/dynamic_relaxation.py:87-128 on K, clamped x=0 face
    row = np.asarray(np.abs(K).sum(axis=1)).ravel()
    dt, sf, c = 1.0, 1.1, 0.1
    mdiag = 0.25 * sf * dt ** 2 * np.maximum(row, 1e-6 * row.max())
    fixed = np.repeat(3 * meshgen.nodes_on_plane(m, 0, "min"), 3) + np.tile([0, 1, 2], len(meshgen.nodes_on_plane(m, 0, "min")))
    minv = 1.0 / mdiag
    minv[fixed] = 0.0
    c1, c2 = (2 - c * dt) / (2 + c * dt), 2 * dt / (2 + c * dt)
    x = np.zeros(n)
    vel = np.zeros(n)
    xd = torch.zeros(n, dtype=torch.float64, device="cuda")
    vd = torch.zeros(n, dtype=torch.float64, device="cuda")
    bd = torch.from_numpy(b).cuda()
    md = torch.from_numpy(minv).cuda()
    rd = torch.zeros(n, dtype=torch.float64, device="cuda")
    for _ in range(50):
        r = b - K @ x
        vel = c1 * vel + c2 * (minv * r)
        x = x + dt * vel
        asm.dr_step(u_d, bd, md, xd, vd, c1, c2, dt, r_out=rd)
    assert rel_2(xd.cpu().numpy(), x) < 1e-11
    assert rel_2(vd.cpu().numpy(), vel) < 1e-11
    assert rel_2(rd.cpu().numpy(), r) < 1e-11
