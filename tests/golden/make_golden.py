"""Generate the golden fixtures in ``tests/golden/`` by running the pSierra reference.

Run in a container that has the reference sources, with ``PSIERRA_REFERENCE_SRC`` set
to the reference's ``src`` directory (the one holding ``psierra/``)::

    PSIERRA_REFERENCE_SRC=<reference>/src python tests/golden/make_golden.py            # all fixtures
    PSIERRA_REFERENCE_SRC=<reference>/src python tests/golden/make_golden.py fbar_box   # one fixture

Every output below comes from the reference's own classes (``Tet4TotalLagrangian``,
``Tet10TotalLagrangian``, ``NeoHookean``, ``SolidDomain``, ``NonlinearStaticAnalysis``,
``DynamicRelaxationAnalysis``) called through their public API; the inputs are
seeded synthetic meshes and fields built with ``psierra_b200.meshgen``.  The GPU
tests read only the ``.npz`` files written here, never the reference.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import _refstub  # noqa: E402

_refstub.install()

from psierra.analysis.dynamic_relaxation import DynamicRelaxationAnalysis  # noqa: E402
from psierra.analysis.nonlinear_dynamic import NonlinearDynamicAnalysis  # noqa: E402
from psierra.analysis.nonlinear_static import NonlinearStaticAnalysis  # noqa: E402
from psierra.damping.rayleigh import RayleighDamping  # noqa: E402
from psierra.boundary.dirichlet import DirichletConstraint, DirichletManager  # noqa: E402
from psierra.boundary.load import NodalForce  # noqa: E402
from psierra.domain.solid import SolidDomain  # noqa: E402
from psierra.element.tet10_total_lagrangian import Tet10TotalLagrangian  # noqa: E402
from psierra.element.tet4_fbar import Tet4Fbar  # noqa: E402
from psierra.element.tet4_total_lagrangian import Tet4TotalLagrangian  # noqa: E402
from psierra.material.neohookean import NeoHookean  # noqa: E402
from psierra.material.parameters import IsotropicElasticParameters  # noqa: E402
from psierra.solver.sparse_linear_solver import ConjugateGradientSolver  # noqa: E402

from psierra_b200 import meshgen  # noqa: E402

DuckMesh = _refstub.DuckMesh


def nh(E, nu, rho=1000.0):
    p = IsotropicElasticParameters()
    p.set_from_youngs_poisson(youngs_modulus=E, poissons_ratio=nu, mass_density=rho)
    return NeoHookean(p)


def random_tets(rng, n, npe):
    """Random well-shaped reference tets (Tet10: straight-edged mid nodes)."""
    base = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], dtype=np.float64)
    out = []
    while len(out) < n:
        s = rng.uniform(0.02, 0.5)
        X = s * (base + rng.normal(0, 0.15, size=(4, 3))) + rng.normal(0, 1.0, size=3)
        d = X[1:] - X[0]
        if np.linalg.det(d) < 0.05 * np.abs(d).max() ** 3:
            continue
        if npe == 10:
            e = [(0, 1), (1, 2), (2, 0), (0, 3), (1, 3), (2, 3)]
            X = np.vstack([X] + [0.5 * (X[a] + X[b])[None] for a, b in e])
        out.append(X)
    return np.stack(out)


def element_fixture(rng, n, npe):
    X = random_tets(rng, n, npe)
    E = rng.uniform(1e3, 1e6, size=n)
    nu = rng.uniform(0.3, 0.49, size=n)
    scale = np.abs(X[:, 1:4] - X[:, 0:1]).max(axis=(1, 2))
    u = rng.normal(0, 1, size=X.shape) * (0.03 * scale)[:, None, None]
    k = np.zeros((n, 3 * npe, 3 * npe))
    f = np.zeros((n, 3 * npe))
    klin = np.zeros_like(k)
    mu = np.zeros(n)
    kap = np.zeros(n)
    lam = np.zeros(n)
    for i in range(n):
        mat = nh(E[i], nu[i])
        el = Tet4TotalLagrangian(mat) if npe == 4 else Tet10TotalLagrangian(mat)
        k[i], f[i] = el.compute_nonlinear_force_and_tangent_stiffness(X[i], u[i])
        klin[i] = el.compute_linear_stiffness_matrix(X[i])
        mu[i] = mat.parameters.shear_modulus
        kap[i] = mat.parameters.bulk_modulus
        lam[i] = mat.parameters.lame_parameter_1
    return dict(X=X, u=u, E=E, nu=nu, mu=mu, kappa=kap, lam=lam, k=k, f=f, k_lin=klin)


def element_extreme_fixture(npe: int = 4, n: int = 40, seed: int = 8):
    """Elements far from element_fixture's states, through the reference's element:
    homogeneous stretch and compression with rotation (det F from 0.35 to 2.5) plus a
    non-homogeneous part, Poisson ratios up to 0.4999, and strains of 1e-7, where the
    reference's stress formula carries its O(mu) cancellation.  Its own random stream,
    so it can be regenerated alone."""
    rng = np.random.default_rng(seed + npe)
    nus = (0.3, 0.45, 0.49, 0.499, 0.4999)
    dets = (0.35, 0.6, 1.8, 2.5)
    keys = ("X", "u", "E", "nu", "mu", "kappa", "lam", "k", "f", "det_F")
    rows = {k: [] for k in keys}
    while len(rows["X"]) < n:
        i = len(rows["X"])
        X = random_tets(rng, 1, npe)[0]
        scale = float(np.abs(X[1:4] - X[0]).max())
        if i % 4 == 3:
            u = rng.normal(0, 1, size=X.shape) * 1e-7 * scale
            det_F = 1.0
        else:
            Rq, _ = np.linalg.qr(rng.normal(size=(3, 3)))
            Qq, _ = np.linalg.qr(rng.normal(size=(3, 3)))
            lam_p = np.exp(rng.normal(0, 0.35, size=3))
            det_F = dets[(i // 4 + i) % len(dets)]
            lam_p *= (det_F / lam_p.prod()) ** (1.0 / 3.0)
            if np.linalg.det(Rq) * np.linalg.det(Qq) < 0:
                Rq[:, 0] = -Rq[:, 0]  # proper rotations only: det F = det_F > 0
            F = Rq @ np.diag(lam_p) @ Qq.T
            c = X[:4].mean(axis=0)
            u = (X - c) @ (F - np.identity(3)).T + rng.normal(0, 0.02 * scale, size=X.shape)
        E = float(rng.uniform(1e3, 1e6))
        nu = nus[i % len(nus)]
        mat = nh(E, nu)
        el = Tet4TotalLagrangian(mat) if npe == 4 else Tet10TotalLagrangian(mat)
        try:
            k, f = el.compute_nonlinear_force_and_tangent_stiffness(X, u)
        except ValueError:
            continue  # the perturbation inverted a quadrature point: draw again
        for key, v in zip(keys, (X, u, E, nu, mat.parameters.shear_modulus, mat.parameters.bulk_modulus,
                                 mat.parameters.lame_parameter_1, k, f, det_F)):
            rows[key].append(v)
    return {k: np.asarray(v) for k, v in rows.items()}


def material_fixture(rng, n=24):
    Fs, Cs, Ss = [], [], []
    for _ in range(n):
        F = np.identity(3) + rng.normal(0, 0.15, size=(3, 3))
        if np.linalg.det(F) <= 0.2:
            continue
        mat = nh(1e4, 0.45)
        C, S = mat.compute_stress_and_tangent(F)
        Fs.append(F), Cs.append(C), Ss.append(S)
    mat = nh(1e4, 0.45)
    return dict(F=np.stack(Fs), C=np.stack(Cs), S=np.stack(Ss),
                mu=mat.parameters.shear_modulus, kappa=mat.parameters.bulk_modulus)


def domain_state(mesh, mat, element, u):
    dom = SolidDomain(DuckMesh(mesh.nodes, mesh.elements), mat, element)
    dom.update_state(u=u.ravel())
    f = dom.assemble_internal_forces()
    K = dom.assemble_tangent_stiffness_matrix()
    Klin = dom.assemble_stiffness_matrix()
    return f, K, Klin


class Tracing(SolidDomain):
    """SolidDomain that records the displacement at every tangent assembly (= Newton iterate)."""

    def __init__(self, *a, **k):
        super().__init__(*a, **k)
        self.trace = []
        self.f_calls = 0

    def assemble_tangent_stiffness_matrix(self):
        self.trace.append(self.u.copy())
        return super().assemble_tangent_stiffness_matrix()

    def assemble_internal_forces(self):
        self.f_calls += 1
        return super().assemble_internal_forces()


def cantilever_problem(mesh, traction):
    clamp = meshgen.nodes_on_plane(mesh, 0, "min")
    dm = DirichletManager(mesh.n_dofs)
    dm.add_constraint(DirichletConstraint(clamp, components=(0, 1, 2), value=0.0))
    f_ext = meshgen.traction_nodal_forces(mesh, 0, "max", [0.0, 0.0, traction])
    return dm, f_ext, clamp


def fbar_fixture():
    """Tet4Fbar (element/tet4_fbar.py) through SolidDomain on a small Kuhn box, plus
    per-element calls with explicit J_bar values."""
    m = meshgen.box_tet4(1.0, 0.5, 0.4, 4, 2, 2)
    u = meshgen.cantilever_seeded_u(m, seed=99) * 3.0
    mat = nh(1e4, 0.45)
    el = Tet4Fbar(mat)
    dom = SolidDomain(DuckMesh(m.nodes, m.elements), mat, el)
    dom.update_state(u=u.ravel())
    f = dom.assemble_internal_forces()
    jbar = el._domain_J_bar.copy()  # J_bar at u (the u = 0 stiffness below resets it)
    K = dom.assemble_tangent_stiffness_matrix()
    Klin = dom.assemble_stiffness_matrix()
    rng = np.random.default_rng(5)
    pick = rng.choice(m.n_elements, size=6, replace=False)
    ke, fe, jb = [], [], []
    for e in pick:
        J_bar = float(jbar[e]) * (1.0 + 0.01 * rng.normal())
        k, fv = Tet4Fbar(mat).compute_nonlinear_force_and_tangent_stiffness(
            m.nodes[m.elements[e]], u.reshape(-1, 3)[m.elements[e]], J_bar=J_bar)
        ke.append(k)
        fe.append(fv)
        jb.append(J_bar)
    return dict(nodes=m.nodes, elements=m.elements, u=u, f=f, K_data=K.data, K_indptr=K.indptr,
                K_indices=K.indices, Klin_data=Klin.data, Klin_indptr=Klin.indptr, Klin_indices=Klin.indices,
                J_bar=jbar, pick=pick, pick_J_bar=np.array(jb), pick_k=np.stack(ke), pick_f=np.stack(fe),
                mu=mat.parameters.shear_modulus, kappa=mat.parameters.bulk_modulus,
                lam=mat.parameters.lame_parameter_1)


def dynamic_fixture():
    """NonlinearDynamicAnalysis (analysis/nonlinear_dynamic.py) on a small cantilever: tip
    traction applied at t = 0, generalized-alpha rho_inf = 0.8, Rayleigh damping, the
    direct linear solver; final u, v, a and the Newton iterations per step."""
    mb = meshgen.box_tet4(1.0, 0.1, 0.1, 8, 2, 2)
    mat = nh(1e5, 0.3, rho=1000.0)
    dm, f_ext, clamp = cantilever_problem(mb, -50.0)
    dom = SolidDomain(DuckMesh(mb.nodes, mb.elements), mat, Tet4TotalLagrangian(mat))
    an = NonlinearDynamicAnalysis(dom, damping=RayleighDamping(0.5, 1e-4), spectral_radius=0.8)
    r = an.solve(dirichlet=dm, f_ext=f_ext, dt=0.05, n_steps=10, nr_iterations=15, nr_tol=1e-8, verbose=False)
    return dict(u=dom.u.copy(), v=dom.v.copy(), a=dom.a.copy(), iterations=np.array(r.iteration_history),
                converged=r.converged, f_ext=f_ext, clamp=clamp, dt=0.05, n_steps=10, rho=1000.0,
                rayleigh=np.array([0.5, 1e-4]), spectral_radius=0.8, nr_tol=1e-8,
                mu=mat.parameters.shear_modulus, kappa=mat.parameters.bulk_modulus,
                lam=mat.parameters.lame_parameter_1)


def dynamic_tet10_fixture():
    """NonlinearDynamicAnalysis with Tet10TotalLagrangian on a small cantilever (6 x 2 x 2
    cells -> 144 Tet10): the same load and integrator settings as dynamic_fixture, plus
    the consistent mass the reference domain assembles (element/tet10_base.py:344-372)."""
    mb = meshgen.tet4_to_tet10(meshgen.box_tet4(1.0, 0.1, 0.1, 6, 2, 2))
    mat = nh(1e5, 0.3, rho=1000.0)
    dm, f_ext, clamp = cantilever_problem(mb, -50.0)
    dom = SolidDomain(DuckMesh(mb.nodes, mb.elements), mat, Tet10TotalLagrangian(mat))
    M = dom.assemble_mass_matrix()
    an = NonlinearDynamicAnalysis(dom, damping=RayleighDamping(0.5, 1e-4), spectral_radius=0.8)
    r = an.solve(dirichlet=dm, f_ext=f_ext, dt=0.05, n_steps=8, nr_iterations=15, nr_tol=1e-8, verbose=False)
    return dict(u=dom.u.copy(), v=dom.v.copy(), a=dom.a.copy(), iterations=np.array(r.iteration_history),
                converged=r.converged, f_ext=f_ext, clamp=clamp, dt=0.05, n_steps=8, rho=1000.0,
                rayleigh=np.array([0.5, 1e-4]), spectral_radius=0.8, nr_tol=1e-8,
                M_data=M.data, M_indptr=M.indptr, M_indices=M.indices)


def tet10_newton_fixture(cells: int = 3, n_steps: int = 8, nr_iterations: int = 20):
    """The Tet10 cube solve at a reduced grid (3^3 cells -> 162 Tet10 by default): clamp
    z = 0, u_z = -0.2 prescribed on z = 1 and ramped over ``n_steps`` increments
    (nonlinear_static.py:271-272), E = 1e4, nu = 0.4, the reference's Newton with its
    direct solver."""
    m = meshgen.tet4_to_tet10(meshgen.box_tet4(1.0, 1.0, 1.0, cells, cells, cells))
    mat = nh(1e4, 0.4)
    bottom = meshgen.nodes_on_plane(m, 2, "min")
    top = meshgen.nodes_on_plane(m, 2, "max")
    dm = DirichletManager(m.n_dofs)
    dm.add_constraint(DirichletConstraint(bottom, components=(0, 1, 2), value=0.0))
    dm.add_constraint(DirichletConstraint(top, components=(2,), value=-0.2))
    dom = SolidDomain(DuckMesh(m.nodes, m.elements), mat, Tet10TotalLagrangian(mat))
    r = NonlinearStaticAnalysis(dom).solve(dirichlet=dm, f_ext=np.zeros(m.n_dofs), n_steps=n_steps,
                                           nr_iterations=nr_iterations, nr_tol=1e-8, verbose=False)
    return dict(u=r.displacement, converged=r.converged, iterations=np.array(r.iteration_history),
                bottom=bottom, top=top, mu=mat.parameters.shear_modulus, kappa=mat.parameters.bulk_modulus,
                cells=cells, n_steps=n_steps)


def tet10_compress6_fixture():
    """The Tet10 compression workload's loading (20 increments of the top-face
    displacement, 30 Newton iterations allowed, tolerance 1e-8) on 6^3 cells -> 1,296
    Tet10: the reference's own Newton converges in 5 iterations per increment."""
    return tet10_newton_fixture(cells=6, n_steps=20, nr_iterations=30)


def main(only=None):
    rng = np.random.default_rng(20261203)
    out = {}
    if only:
        # fixtures that need no shared random stream can be regenerated on their own
        gens = {"fbar_box": fbar_fixture, "dynamic_beam": dynamic_fixture, "tet10_newton": tet10_newton_fixture,
                "tet10_compress6": tet10_compress6_fixture,
                "dynamic_tet10": dynamic_tet10_fixture,
                "element_extreme_tet4": lambda: element_extreme_fixture(4),
                "element_extreme_tet10": lambda: element_extreme_fixture(10, n=20)}
        for name in only:
            out[name] = gens[name]()
        for name, d in out.items():
            path = os.path.join(HERE, f"{name}.npz")
            np.savez_compressed(path, **d)
            print(f"{name}: {os.path.getsize(path) / 1024:.1f} KiB")
        return

    out["element_tet4"] = element_fixture(rng, 64, 4)
    out["element_tet10"] = element_fixture(rng, 16, 10)
    out["material_nh"] = material_fixture(rng)

    # cfg1 seeded state: cantilever 1.0 x 0.1 x 0.1, 40x4x4 Kuhn, E=1e5, nu=0.3.
    m1 = meshgen.box_tet4(1.0, 0.1, 0.1, 40, 4, 4)
    u1 = meshgen.cantilever_seeded_u(m1, seed=1234)
    mat1 = nh(1e5, 0.3)
    f1, K1, Kl1 = domain_state(m1, mat1, Tet4TotalLagrangian(mat1), u1)
    out["cfg1_seeded"] = dict(seed=1234, u=u1, f=f1, K_data=K1.data, K_indptr=K1.indptr,
                              K_indices=K1.indices, Klin_data=Kl1.data,
                              mu=mat1.parameters.shear_modulus, kappa=mat1.parameters.bulk_modulus,
                              lam=mat1.parameters.lame_parameter_1)

    # Small Tet10 box (3x3x3 cells -> 162 quadratic tets), E=1e4, nu=0.4.
    m10 = meshgen.tet4_to_tet10(meshgen.box_tet4(1.0, 1.0, 1.0, 3, 3, 3))
    u10 = meshgen.cube_smooth_u(m10, seed=77) * 2.0
    mat10 = nh(1e4, 0.4)
    f10, K10, Kl10 = domain_state(m10, mat10, Tet10TotalLagrangian(mat10), u10)
    out["tet10_box3"] = dict(seed=77, nodes=m10.nodes, elements=m10.elements, u=u10, f=f10,
                             K_data=K10.data, K_indptr=K10.indptr, K_indices=K10.indices,
                             Klin_data=Kl10.data,
                             mu=mat10.parameters.shear_modulus, kappa=mat10.parameters.bulk_modulus,
                             lam=mat10.parameters.lame_parameter_1)

    # Newton on the 5-tet unit cube (reference test_analysis_nonlinear.py:28-70 setup).
    cube_nodes = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                           [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], dtype=np.float64)
    cube_tets = np.array([[0, 1, 3, 4], [1, 2, 3, 6], [1, 4, 5, 6], [3, 4, 6, 7], [1, 3, 4, 6]])
    cube = meshgen.TetMesh(cube_nodes, cube_tets)
    mat_c = nh(10e3, 0.45)
    res = {}
    for total_fz, n_steps, tol in ((50.0, 4, 1e-4), (15.0, 5, 1e-5)):
        dom = Tracing(DuckMesh(cube_nodes, cube_tets), mat_c, Tet4TotalLagrangian(mat_c))
        fixed = meshgen.nodes_on_plane(cube, 2, "min")
        top = meshgen.nodes_on_plane(cube, 2, "max")
        dm = DirichletManager(cube.n_dofs)
        dm.add_constraint(DirichletConstraint(fixed, components=(0, 1, 2), value=0.0))
        f_ext = NodalForce(top, [0.0, 0.0, total_fz / len(top)]).compute_force_vector(cube.n_dofs)
        r = NonlinearStaticAnalysis(dom).solve(dirichlet=dm, f_ext=f_ext, n_steps=n_steps,
                                               nr_iterations=15, nr_tol=tol, verbose=False)
        key = f"fz{int(total_fz)}"
        res[f"{key}_u"] = r.displacement
        res[f"{key}_reactions"] = r.reactions
        res[f"{key}_iterations"] = np.array(r.iteration_history)
        res[f"{key}_trace"] = np.stack(dom.trace)
        res[f"{key}_f_ext"] = f_ext
        res[f"{key}_fixed"] = fixed
        res[f"{key}_n_steps"] = n_steps
        res[f"{key}_tol"] = tol
        if total_fz == 15.0:
            dr_dom = SolidDomain(DuckMesh(cube_nodes, cube_tets), mat_c, Tet4TotalLagrangian(mat_c))
            dr = DynamicRelaxationAnalysis(dr_dom, damping_type="kinetic", safety_factor=1.2, dt=1.0)
            drr = dr.solve(dirichlet=dm, f_ext=f_ext, tol=1e-4, max_steps=1000, verbose=False)
            res["dr_kinetic_u"] = drr.displacement
            res["dr_kinetic_steps"] = drr.steps_completed
            res["dr_kinetic_peaks"] = drr.kinetic_peaks
            res["dr_kinetic_history"] = np.array(drr.residual_history)
    res["mu"] = mat_c.parameters.shear_modulus
    res["kappa"] = mat_c.parameters.bulk_modulus
    res["lam"] = mat_c.parameters.lame_parameter_1
    out["newton_cube"] = res

    # Cantilever beam Newton that converges (10x2x2 cells, traction -20 Pa, 4 increments),
    # and the first iterates of the cfg1 problem as specified (-500 Pa, 10 increments).
    mb = meshgen.box_tet4(1.0, 0.1, 0.1, 10, 2, 2)
    mat_b = nh(1e5, 0.3)
    dm, f_ext, clamp = cantilever_problem(mb, -20.0)
    dom = Tracing(DuckMesh(mb.nodes, mb.elements), mat_b, Tet4TotalLagrangian(mat_b))
    r = NonlinearStaticAnalysis(dom).solve(dirichlet=dm, f_ext=f_ext, n_steps=4,
                                           nr_iterations=25, nr_tol=1e-8, verbose=False)
    beam = dict(u=r.displacement, converged=r.converged, iterations=np.array(r.iteration_history),
                trace=np.stack(dom.trace), f_ext=f_ext, clamp=clamp, reactions=r.reactions,
                mu=mat_b.parameters.shear_modulus, kappa=mat_b.parameters.bulk_modulus,
                lam=mat_b.parameters.lame_parameter_1)
    # Same beam solved with the reference Jacobi-CG linear solver.
    dom2 = Tracing(DuckMesh(mb.nodes, mb.elements), mat_b, Tet4TotalLagrangian(mat_b))
    r2 = NonlinearStaticAnalysis(dom2, linear_solver=ConjugateGradientSolver(tolerance=1e-10, max_iterations=5000)).solve(
        dirichlet=dm, f_ext=f_ext, n_steps=4, nr_iterations=25, nr_tol=1e-8, verbose=False)
    beam["cg_u"] = r2.displacement
    beam["cg_iterations"] = np.array(r2.iteration_history)

    # Viscous dynamic relaxation on the same beam, c = 0.1, 400 pseudo-steps.
    dr_dom = SolidDomain(DuckMesh(mb.nodes, mb.elements), mat_b, Tet4TotalLagrangian(mat_b))
    drv = DynamicRelaxationAnalysis(dr_dom, damping_type="viscous", viscous_damping=0.1,
                                    safety_factor=1.1, dt=1.0)
    dres = drv.solve(dirichlet=dm, f_ext=f_ext, tol=1e-12, max_steps=400, min_steps=10, verbose=False)
    beam["dr_viscous_u"] = dres.displacement
    beam["dr_viscous_history"] = np.array(dres.residual_history)
    beam["dr_viscous_steps"] = dres.steps_completed
    out["newton_beam"] = beam

    m1b = meshgen.box_tet4(1.0, 0.1, 0.1, 40, 4, 4)
    dm1, f1e, clamp1 = cantilever_problem(m1b, -500.0)
    dom1 = Tracing(DuckMesh(m1b.nodes, m1b.elements), mat1, Tet4TotalLagrangian(mat1))
    r1 = NonlinearStaticAnalysis(dom1).solve(dirichlet=dm1, f_ext=f1e, n_steps=10,
                                             nr_iterations=3, nr_tol=1e-4, verbose=False)
    out["cfg1_newton"] = dict(trace=np.stack(dom1.trace), f_ext=f1e, clamp=clamp1,
                              converged=r1.converged, f_calls=dom1.f_calls)

    out["fbar_box"] = fbar_fixture()
    out["dynamic_beam"] = dynamic_fixture()
    out["tet10_newton"] = tet10_newton_fixture()
    out["tet10_compress6"] = tet10_compress6_fixture()
    out["dynamic_tet10"] = dynamic_tet10_fixture()
    out["element_extreme_tet4"] = element_extreme_fixture(4)
    out["element_extreme_tet10"] = element_extreme_fixture(10, n=20)

    for name, d in out.items():
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **d)
        print(f"{name}: {os.path.getsize(path) / 1024:.1f} KiB")


if __name__ == "__main__":
    main(sys.argv[1:] or None)
