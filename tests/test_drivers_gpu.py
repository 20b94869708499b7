"""The GPU element driven by the Newton and dynamic-relaxation drivers, against the
reference's own runs of the same problems (golden traces from pSierra's
NonlinearStaticAnalysis / DynamicRelaxationAnalysis with its CPU element)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden, rel_2, rel_max
from oracle.assembly import assemble_mass
from psierra_b200 import meshgen
from psierra_b200.analysis import DynamicRelaxationAnalysis, NonlinearStaticAnalysis
from psierra_b200.domain import DirichletConstraint, DirichletManager, SolidDomain
from psierra_b200.element import Tet4TotalLagrangian
from psierra_b200.material import IsotropicElasticParameters, NeoHookean
from psierra_b200.solver import ConjugateGradientSolver

pytestmark = pytest.mark.gpu

CUBE_NODES = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]],
                      dtype=np.float64)
CUBE_TETS = np.array([[0, 1, 3, 4], [1, 2, 3, 6], [1, 4, 5, 6], [3, 4, 6, 7], [1, 3, 4, 6]])


def nh(E, nu, rho=1000.0):
    p = IsotropicElasticParameters()
    p.set_from_youngs_poisson(youngs_modulus=E, poissons_ratio=nu, mass_density=rho)
    return NeoHookean(p)


def clamp_manager(mesh, nodes):
    dm = DirichletManager(mesh.n_dofs)
    dm.add_constraint(DirichletConstraint(nodes, components=(0, 1, 2), value=0.0))
    return dm


class Tracing(SolidDomain):
    def __init__(self, *a, **k):
        super().__init__(*a, **k)
        self.trace = []

    def assemble_tangent_stiffness_matrix(self):
        self.trace.append(self.u.copy())
        return super().assemble_tangent_stiffness_matrix()


@pytest.mark.parametrize("key,n_steps,tol", [("fz50", 4, 1e-4), ("fz15", 5, 1e-5)])
def test_newton_cube_matches_reference(key, n_steps, tol):
    g = golden("newton_cube")
    cube = meshgen.TetMesh(CUBE_NODES, CUBE_TETS)
    mat = nh(10e3, 0.45)
    dom = Tracing(cube, mat, Tet4TotalLagrangian(mat))
    r = NonlinearStaticAnalysis(dom).solve(clamp_manager(cube, g[f"{key}_fixed"]), f_ext=g[f"{key}_f_ext"],
                                           n_steps=n_steps, nr_iterations=15, nr_tol=tol)
    assert r.converged and r.steps_completed == n_steps
    assert list(r.iteration_history) == list(g[f"{key}_iterations"])
    trace = np.stack(dom.trace)
    assert trace.shape == g[f"{key}_trace"].shape
    # measured: trace <= 9.4e-14, u <= 8.3e-14, reactions <= 3.0e-13
    assert rel_max(trace, g[f"{key}_trace"]) < 1e-12
    assert rel_2(r.displacement, g[f"{key}_u"]) < 1e-12
    assert rel_max(r.reactions, g[f"{key}_reactions"]) < 1e-11


def test_dynamic_relaxation_kinetic_cube_matches_reference():
    g = golden("newton_cube")
    cube = meshgen.TetMesh(CUBE_NODES, CUBE_TETS)
    mat = nh(10e3, 0.45)
    dom = SolidDomain(cube, mat, Tet4TotalLagrangian(mat))
    dr = DynamicRelaxationAnalysis(dom, damping_type="kinetic", safety_factor=1.2, dt=1.0)
    r = dr.solve(clamp_manager(cube, g["fz15_fixed"]), f_ext=g["fz15_f_ext"], tol=1e-4, max_steps=1000)
    assert r.converged
    assert r.steps_completed == int(g["dr_kinetic_steps"]) and r.kinetic_peaks == int(g["dr_kinetic_peaks"])
    # measured: u 6.5e-14, residual history 2.3e-12
    assert rel_2(r.displacement, g["dr_kinetic_u"]) < 1e-12
    assert rel_max(np.array(r.residual_history), g["dr_kinetic_history"]) < 1e-10


@pytest.mark.parametrize("solver", ["direct", "gpu-cg"])
def test_newton_beam_matches_reference(solver):
    g = golden("newton_beam")
    mb = meshgen.box_tet4(1.0, 0.1, 0.1, 10, 2, 2)
    mat = nh(1e5, 0.3)
    dom = Tracing(mb, mat, Tet4TotalLagrangian(mat))
    lin = ConjugateGradientSolver(tolerance=1e-10, max_iterations=5000) if solver == "gpu-cg" else None
    r = NonlinearStaticAnalysis(dom, linear_solver=lin).solve(clamp_manager(mb, g["clamp"]), f_ext=g["f_ext"],
                                                              n_steps=4, nr_iterations=25, nr_tol=1e-8)
    assert r.converged
    ref_u = g["u"] if solver == "direct" else g["cg_u"]
    ref_it = g["iterations"] if solver == "direct" else g["cg_iterations"]
    assert list(r.iteration_history) == list(ref_it)
    assert rel_2(r.displacement, ref_u) < 1e-12  # measured 3.4e-14 (direct), 3.2e-14 (GPU CG)
    if solver == "direct":
        assert rel_max(np.stack(dom.trace), g["trace"]) < 1e-11  # measured 2.6e-13


def test_dynamic_relaxation_viscous_beam_matches_reference():
    g = golden("newton_beam")
    mb = meshgen.box_tet4(1.0, 0.1, 0.1, 10, 2, 2)
    mat = nh(1e5, 0.3)
    dom = SolidDomain(mb, mat, Tet4TotalLagrangian(mat))
    dr = DynamicRelaxationAnalysis(dom, damping_type="viscous", viscous_damping=0.1, safety_factor=1.1, dt=1.0)
    r = dr.solve(clamp_manager(mb, g["clamp"]), f_ext=g["f_ext"], tol=1e-12, max_steps=400, min_steps=10)
    assert r.steps_completed == int(g["dr_viscous_steps"])
    # measured: u 1.5e-13, residual history 1.4e-11 (its late entries are residuals near the
    # 1e-12 stopping tolerance, where the reference's own f_int rounding is a visible share)
    assert rel_2(r.displacement, g["dr_viscous_u"]) < 1e-12
    assert rel_max(np.array(r.residual_history), g["dr_viscous_history"]) < 5e-10


def test_cfg1_first_newton_iterates_match_reference():
    g = golden("cfg1_newton")
    m = meshgen.box_tet4(1.0, 0.1, 0.1, 40, 4, 4)
    mat = nh(1e5, 0.3)
    dom = Tracing(m, mat, Tet4TotalLagrangian(mat))
    r = NonlinearStaticAnalysis(dom).solve(clamp_manager(m, g["clamp"]), f_ext=g["f_ext"], n_steps=10,
                                           nr_iterations=3, nr_tol=1e-4)
    assert not r.converged and bool(g["converged"]) is False
    trace = np.stack(dom.trace)
    assert trace.shape == g["trace"].shape
    # measured 4.3e-11: these iterates do not converge, and the tangent's condition number
    # (~2e6) amplifies the reference's own O(mu) rounding of f_int (~1e-13 relative)
    assert rel_max(trace, g["trace"]) < 1e-9


def test_mass_matrix_matches_oracle():
    m = meshgen.box_tet4(1.0, 0.3, 0.2, 6, 3, 2)
    mat = nh(1e5, 0.3, rho=1040.0)
    M = Tet4TotalLagrangian(mat).assemble_mass_matrix(m)
    Mo = assemble_mass(m.nodes, m.elements, 1040.0)
    assert np.array_equal(M.indptr, Mo.indptr) and np.array_equal(M.indices, Mo.indices)
    assert rel_max(M.data, Mo.data) < 1e-14
