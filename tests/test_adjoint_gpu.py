"""Adjoint gradients against central finite differences (GPU).

Tolerance: 1e-5 relative (the north-star bound for adjoint gradients vs FD).
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import golden, rel_2
from psierra_b200 import meshgen
from psierra_b200.adjoint import internal_force, static_equilibrium
from psierra_b200.assembler import GPUAssembler
from psierra_b200.material import NeoHookeanField
from psierra_b200.newton import DeviceNewton

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda")


def problem(seed=0, cells=(3, 2, 2)):
    m = meshgen.box_tet4(1.0, 0.4, 0.3, *cells)
    rng = np.random.default_rng(seed)
    mu = np.exp(np.log(1000.0) + 0.3 * rng.normal(size=m.n_elements))
    kappa = 50.0 * mu
    asm = GPUAssembler(m.nodes, m.elements, NeoHookeanField(mu, kappa))
    return m, asm, mu, kappa, rng


def test_internal_force_vjp_matches_central_differences():
    m, asm, mu, kappa, rng = problem()
    X = torch.from_numpy(m.nodes.copy()).to(DEV).requires_grad_(True)
    u = torch.from_numpy(0.03 * rng.normal(size=(m.n_nodes, 3))).to(DEV).requires_grad_(True)
    mu_t = torch.from_numpy(mu).to(DEV).requires_grad_(True)
    ka_t = torch.from_numpy(kappa).to(DEV).requires_grad_(True)
    w = torch.from_numpy(rng.normal(size=m.n_dofs)).to(DEV)
    f = internal_force(asm, X, u, mu_t, ka_t)
    (f @ w).backward()

    def F(Xn, un, mun, kan):
        with torch.no_grad():
            return float(internal_force(asm, Xn, un, mun, kan) @ w)

    h = 1e-6
    for name, t, scale in (("X", X, 1.0), ("u", u, 1.0), ("mu", mu_t, 1000.0), ("kappa", ka_t, 50000.0)):
        g = t.grad.detach().reshape(-1)
        idx = rng.choice(g.numel(), size=8, replace=False)
        fd = []
        for i in idx:
            args = [X.detach().clone(), u.detach().clone(), mu_t.detach().clone(), ka_t.detach().clone()]
            k = ("X", "u", "mu", "kappa").index(name)
            step = h * scale
            args[k].view(-1)[i] += step
            fp = F(*args)
            args[k].view(-1)[i] -= 2 * step
            fm = F(*args)
            fd.append((fp - fm) / (2 * step))
        fd = np.array(fd)
        got = g[torch.as_tensor(idx, device=DEV)].cpu().numpy()
        assert np.abs(got - fd).max() <= 1e-5 * np.abs(fd).max() + 1e-12, name


def test_static_equilibrium_gradient_matches_central_differences():
    m, asm, mu, kappa, rng = problem(seed=3, cells=(6, 2, 2))
    clamp = meshgen.nodes_on_plane(m, 0, "min")
    fixed = np.concatenate([3 * clamp + c for c in range(3)])
    nt = DeviceNewton(asm, fixed, precision="fp64", pcg_tol=1e-13)
    f_ext = torch.from_numpy(meshgen.traction_nodal_forces(m, 0, "max", [0.0, 0.0, -8.0])).to(DEV)
    obs = np.arange(m.n_dofs)[2::3]
    tgt = torch.zeros(len(obs), dtype=torch.float64, device=DEV)
    obs_t = torch.from_numpy(obs).to(DEV)

    def loss_of(mu_np):
        mt = torch.from_numpy(mu_np).to(DEV).requires_grad_(True)
        u = static_equilibrium(nt, mt, 50.0 * mt, f_ext, n_steps=2, nr_tol=1e-10, polish=3)
        L = 0.5 * torch.sum((u[obs_t] - tgt) ** 2)
        return L, mt

    L, mt = loss_of(mu)
    L.backward()
    g = mt.grad.cpu().numpy()
    for e in rng.choice(m.n_elements, size=8, replace=False):
        h = 1e-4 * mu[e]
        mp, mm = mu.copy(), mu.copy()
        mp[e] += h
        mm[e] -= h
        with torch.no_grad():
            fd = (float(loss_of(mp)[0]) - float(loss_of(mm)[0])) / (2 * h)
        assert abs(g[e] - fd) <= 1e-5 * abs(fd) + 1e-14 * abs(float(L)), (e, g[e], fd)


def test_device_newton_matches_reference_beam():
    g = golden("newton_beam")
    mb = meshgen.box_tet4(1.0, 0.1, 0.1, 10, 2, 2)
    mu, kappa = float(g["mu"]), float(g["kappa"])
    E = mb.n_elements
    asm = GPUAssembler(mb.nodes, mb.elements, NeoHookeanField(np.full(E, mu), np.full(E, kappa)))
    fixed = np.concatenate([3 * g["clamp"] + c for c in range(3)])
    nt = DeviceNewton(asm, fixed, precision="fp64", pcg_tol=1e-13)
    res = nt.solve(torch.from_numpy(g["f_ext"]).to(DEV), n_steps=4, nr_iterations=25, nr_tol=1e-8)
    assert res.converged
    assert rel_2(res.u.cpu().numpy(), g["u"]) < 1e-8
    # the FP32-mixed tangent converges to the same FP64 equilibrium
    nt32 = DeviceNewton(asm, fixed, precision="fp32-mixed", pcg_tol=1e-10)
    r32 = nt32.solve(torch.from_numpy(g["f_ext"]).to(DEV), n_steps=4, nr_iterations=40, nr_tol=1e-8)
    assert r32.converged
    assert rel_2(r32.u.cpu().numpy(), g["u"]) < 1e-7


def test_shear_modulus_identification_lowers_the_misfit():
    from psierra_b200.adjoint import identify_shear_moduli

    m, asm, mu_true, _, rng = problem(seed=5, cells=(4, 2, 2))
    clamp = meshgen.nodes_on_plane(m, 0, "min")
    fixed = np.concatenate([3 * clamp + c for c in range(3)])
    nt = DeviceNewton(asm, fixed, precision="fp64", pcg_tol=1e-12)
    f_ext = torch.from_numpy(meshgen.traction_nodal_forces(m, 0, "max", [0.0, 0.0, -8.0])).to(DEV)
    with torch.no_grad():
        mt = torch.from_numpy(mu_true).to(DEV)
        u_true = static_equilibrium(nt, mt, 50.0 * mt, f_ext, n_steps=1).cpu().numpy()
    obs = np.setdiff1d(np.arange(m.n_dofs), fixed)
    mu0 = np.full(m.n_elements, float(np.exp(np.mean(np.log(mu_true)))))
    mu_fit, hist = identify_shear_moduli(nt, f_ext, obs, u_true[obs], mu0, max_iter=15)
    # 96 per-element moduli from one load case: under-determined, so only the misfit is checked
    assert min(hist) < 0.2 * hist[0]
    assert np.all(np.isfinite(mu_fit)) and np.all(mu_fit > 0)


def test_ellipsoid_gravity_identification_gradient():
    """The ellipsoid workload at a coarse spacing: gravity through the consistent mass,
    clamp z < -0.06, mu_e ~ LogNormal(ln 1000, 0.3), kappa = 50 mu; the gradient of the
    displacement misfit against a second seed's solution, checked by central differences
    (h = 1e-4 mu_e) on random elements.  Loaded to 20 % of gravity: the soft body resting
    on its small clamped cap loses static stability (it starts to tip) near a third of
    the full load, where no nearby equilibrium exists for Newton to find."""
    import scipy.sparse as spsp

    m = meshgen.ellipsoid_tet4(0.08, 0.06, 0.07, 0.012)
    rng = np.random.default_rng(41)
    mu_t = np.exp(np.log(1000.0) + 0.3 * rng.normal(size=m.n_elements))
    mu0 = np.exp(np.log(1000.0) + 0.3 * np.random.default_rng(42).normal(size=m.n_elements))
    asm = GPUAssembler(m.nodes, m.elements, NeoHookeanField(mu0, 50.0 * mu0, mass_density=1040.0))
    _, mv = asm.assemble(None, mass=True)
    M = spsp.csr_matrix((mv.cpu().numpy(), asm.pattern.indices, asm.pattern.indptr), shape=(m.n_dofs,) * 2)
    gvec = np.tile([0.0, 0.0, -9.81], m.n_nodes)
    f_ext = torch.from_numpy(0.2 * (M @ gvec)).to(DEV)
    fixed_nodes = np.where(m.nodes[:, 2] < -0.06 + 1e-12)[0]
    assert fixed_nodes.size > 3
    fixed = np.concatenate([3 * fixed_nodes + c for c in range(3)])
    nt = DeviceNewton(asm, fixed, precision="fp64", pcg_tol=1e-13)
    with torch.no_grad():
        mt = torch.from_numpy(mu_t).to(DEV)
        u_tgt = static_equilibrium(nt, mt, 50.0 * mt, f_ext, n_steps=2, polish=3)

    def loss_of(mu_np):
        mv_ = torch.from_numpy(mu_np).to(DEV).requires_grad_(True)
        u = static_equilibrium(nt, mv_, 50.0 * mv_, f_ext, n_steps=2, polish=3)
        return 0.5 * torch.sum((u - u_tgt) ** 2), mv_

    L, mv_ = loss_of(mu0)
    L.backward()
    g = mv_.grad.cpu().numpy()
    for e in rng.choice(m.n_elements, size=8, replace=False):
        h = 1e-4 * mu0[e]
        mp, mm = mu0.copy(), mu0.copy()
        mp[e] += h
        mm[e] -= h
        with torch.no_grad():
            fd = (float(loss_of(mp)[0]) - float(loss_of(mm)[0])) / (2 * h)
        assert abs(g[e] - fd) <= 1e-5 * abs(fd) + 1e-12 * abs(float(L.detach())), (e, g[e], fd)


def test_adjoint_parameter_derivatives_match_the_reference_element():
    """w . df/dmu_e and w . df/dkappa_e of the adjoint kernel against the reference
    element's force at (mu, kappa) = (1, 0) and (0, 1): the NeoHookean stress is linear in
    the moduli at fixed F (material/neohookean.py:87-114), so these are the exact
    derivatives of the reference's f_int."""
    from oracle import equilibrium

    m, asm, mu, kappa, rng = problem(seed=9, cells=(4, 3, 2))
    u = 0.03 * rng.normal(size=(m.n_nodes, 3))
    w = rng.normal(size=m.n_dofs)
    _, gmu, gka = asm.adjoint(torch.from_numpy(u.reshape(-1)).to(DEV), torch.from_numpy(w).to(DEV))
    rmu, rka = equilibrium.force_parameter_gradients(m.nodes, m.elements, u, w)
    assert np.abs(gmu.cpu().numpy() - rmu).max() <= 1e-11 * np.abs(rmu).max()
    assert np.abs(gka.cpu().numpy() - rka).max() <= 1e-11 * np.abs(rka).max()


def test_equilibrium_gradient_matches_reference_forward_model():
    """dL/dmu_e through StaticEquilibrium (device Newton + adjoint PCG) against central
    differences h = 1e-6 mu_e of the reference forward model: the oracle's Newton with the
    direct solver on the reference element and assembly (oracle/equilibrium.py, pinned to
    the reference's own Newton run), the way the reference identifies parameters
    (inverse/parameter_identification.py:346-383).  kappa = 50 mu moves with mu; the target
    displacement comes from a second seeded mu field; 32 random elements; 1e-5 relative."""
    from oracle import equilibrium

    m, asm, mu, kappa, rng = problem(seed=13, cells=(4, 2, 2))
    clamp = meshgen.nodes_on_plane(m, 0, "min")
    fixed = np.concatenate([3 * clamp + c for c in range(3)])
    f_np = meshgen.traction_nodal_forces(m, 0, "max", [0.0, 0.0, -8.0])
    f_ext = torch.from_numpy(f_np).to(DEV)
    mu_tgt = np.exp(np.log(1000.0) + 0.3 * np.random.default_rng(14).normal(size=m.n_elements))
    u_tgt = equilibrium.solve_static(m.nodes, m.elements, mu_tgt, 50.0 * mu_tgt, fixed, f_np)
    obs = np.setdiff1d(np.arange(m.n_dofs), fixed)

    def ref_loss(mu_np):
        u = equilibrium.solve_static(m.nodes, m.elements, mu_np, 50.0 * mu_np, fixed, f_np)
        return 0.5 * float(np.sum((u[obs] - u_tgt[obs]) ** 2))

    nt = DeviceNewton(asm, fixed, precision="fp64", pcg_tol=1e-13)
    mt = torch.from_numpy(mu).to(DEV).requires_grad_(True)
    u = static_equilibrium(nt, mt, 50.0 * mt, f_ext, n_steps=2, nr_tol=1e-12, polish=3)
    obs_t = torch.from_numpy(obs).to(DEV)
    L = 0.5 * torch.sum((u[obs_t] - torch.from_numpy(u_tgt[obs]).to(DEV)) ** 2)
    L.backward()
    g = mt.grad.cpu().numpy()
    assert abs(float(L.detach()) - ref_loss(mu)) <= 1e-8 * ref_loss(mu)
    for e in rng.choice(m.n_elements, size=32, replace=False):
        h = 1e-6 * mu[e]
        mp, mm = mu.copy(), mu.copy()
        mp[e] += h
        mm[e] -= h
        fd = (ref_loss(mp) - ref_loss(mm)) / (2 * h)
        assert abs(g[e] - fd) <= 1e-5 * abs(fd) + 1e-12 * float(L.detach()) / mu[e], (e, g[e], fd)
