"""Host logic of the drivers with an analytic fake domain (no GPU), in the manner of the
reference's SpringDomain tests (psierra tests/test_analysis_solver_foundation.py)."""
from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse as spsp

from psierra_b200.analysis import ContactAwareLineSearch, NonlinearStaticAnalysis, is_element_inversion_error
from psierra_b200.domain import DirichletManager


class SpringDomain:
    """Two hardening springs in series: f_int = k (u + u^3) per spring (exact tangent)."""

    def __init__(self, k=10.0):
        self.k = k
        self.u = np.zeros(3)
        self.v = np.zeros(3)
        self.a = np.zeros(3)
        self.n_dofs = 3

    def update_state(self, u=None, v=None, a=None):
        if u is not None:
            self.u[:] = u

    def commit_state(self):
        pass

    def _e(self):
        return np.diff(self.u)

    def assemble_internal_forces(self):
        e = self._e()
        s = self.k * (e + e ** 3)
        f = np.zeros(3)
        f[:2] -= s
        f[1:] += s
        return f

    def assemble_tangent_stiffness_matrix(self):
        e = self._e()
        kk = self.k * (1 + 3 * e ** 2)
        K = np.zeros((3, 3))
        for i, c in enumerate(kk):
            K[i:i + 2, i:i + 2] += c * np.array([[1, -1], [-1, 1]])
        return spsp.csr_matrix(K)


def test_newton_converges_quadratically_on_springs():
    dom = SpringDomain()
    dm = DirichletManager(3)
    from psierra_b200.domain import DirichletConstraint

    dm.add_constraint(DirichletConstraint([0], components=(0,), value=0.0, dofs_per_node=1))
    f = np.array([0.0, 0.0, 25.0])
    r = NonlinearStaticAnalysis(dom).solve(dm, f_ext=f, n_steps=2, nr_iterations=20, nr_tol=1e-12)
    assert r.converged and r.steps_completed == 2
    e = np.diff(r.displacement)
    assert np.allclose(10.0 * (e + e ** 3), 25.0, rtol=1e-10)
    assert np.allclose(r.reactions[1:], 0.0, atol=1e-9)


def test_line_search_rules():
    ls = ContactAwareLineSearch()
    # strict decrease at the full step
    assert ls.search(lambda a: 0.5, 1.0, 1e-9).alpha == 1.0
    # inversion at the full step, decrease at half
    def f(a):
        if a > 0.6:
            raise ValueError("Element inversion detected: det(F) = -1.0000e-01 <= 0.")
        return 0.9
    r = ls.search(f, 1.0, 1e-9)
    assert r.success and r.alpha == 0.5 and r.element_inversion_encountered
    # no admissible trial at all
    def g(a):
        raise ValueError("Element inversion detected: det(F) = -1.0000e-01 <= 0.")
    r = ls.search(g, 1.0, 1e-9)
    assert not r.success and "inversion" in r.rejection_reason
    # unrelated errors propagate
    with pytest.raises(KeyError):
        ls.search(lambda a: (_ for _ in ()).throw(KeyError("x")), 1.0, 1e-9)
    assert is_element_inversion_error(ValueError("Element inversion detected: det(F) = 0 <= 0."))
    assert not is_element_inversion_error(ValueError("something else"))


def test_concat_meshes_offsets_and_beam_batch_ranges():
    from psierra_b200 import meshgen

    ms = [meshgen.box_tet4(1.0, 0.1, 0.1, n, 1, 1) for n in (2, 5, 3)]
    u, no, eo = meshgen.concat_meshes(ms)
    assert list(no) == [0, 12, 36, 52] and list(eo) == [0, 12, 42, 60]
    assert np.array_equal(u.elements[12:42], ms[1].elements + 12)
    assert np.array_equal(u.nodes[36:52], ms[2].nodes)
    b = meshgen.beam_batch(n=32, target_tets=2e5, seed=1)
    tot = sum(c.mesh.n_elements for c in b)
    assert abs(tot - 2e5) < 0.05 * 2e5
    for c in b:
        nx, ny, nz = c.cells
        assert 8 <= nx <= 120 and 2 <= ny <= 10 and ny == nz
        assert 0.5 <= c.length <= 2.0 and 1e3 <= c.youngs <= 1e6 and 0.3 <= c.poisson <= 0.49
        assert 10.0 <= c.traction[0] <= 1000.0 and c.traction[2] <= 0.0
        assert 400.0 * -c.traction[2] * c.length ** 2 / c.youngs <= 0.25 + 1e-12


class MassSpringDomain(SpringDomain):
    """SpringDomain with the small-strain stiffness and a diagonal mass, as the dynamic
    relaxation driver needs them."""

    def __init__(self, k=10.0, masses=(2.0, 1.0, 0.5)):
        super().__init__(k)
        self.masses = np.asarray(masses, dtype=np.float64)

    def assemble_stiffness_matrix(self):
        K = np.zeros((3, 3))
        for i in range(2):
            K[i:i + 2, i:i + 2] += self.k * np.array([[1, -1], [-1, 1]])
        return spsp.csr_matrix(K)

    def assemble_mass_matrix(self):
        return spsp.diags(self.masses).tocsr()


def _spring_dirichlet():
    from psierra_b200.domain import DirichletConstraint

    dm = DirichletManager(3)
    dm.add_constraint(DirichletConstraint([0], components=(0,), value=0.0, dofs_per_node=1))
    return dm


@pytest.mark.parametrize("mass", ["gerschgorin", "lumped"])
def test_dynamic_relaxation_mass_options_reach_the_equilibrium(mass):
    from psierra_b200.analysis import DynamicRelaxationAnalysis

    # a load at which the springs stiffen by 17%: within the margin of safety factor 2
    # (the masses come from the small-strain stiffness)
    f = np.array([0.0, 0.0, 2.5])
    dr = DynamicRelaxationAnalysis(MassSpringDomain(), damping_type="viscous", viscous_damping=0.3, dt=1.0,
                                   safety_factor=2.0, mass=mass)
    r = dr.solve(_spring_dirichlet(), f_ext=f, tol=1e-10, max_steps=20000)
    assert r.converged
    e = np.diff(r.displacement)
    assert np.allclose(10.0 * (e + e ** 3), 2.5, rtol=1e-8)


def test_lumped_mass_takes_the_rows_of_the_mass_matrix_and_a_stable_step():
    from psierra_b200.analysis import DynamicRelaxationAnalysis

    dom = MassSpringDomain()
    free, fixed = np.array([1, 2]), np.array([0])
    rows = np.array([20.0, 40.0, 20.0])  # absolute row sums of the small-strain stiffness
    for sf in (1.1, 2.0):
        m, inv, dt = DynamicRelaxationAnalysis(dom, safety_factor=sf, dt=10.0, mass="lumped").fictitious_mass(
            10.0, free, fixed)
        assert np.array_equal(m, dom.masses) and inv[0] == 0.0 and np.allclose(inv[1:], 1.0 / dom.masses[1:])
        # 2 / sqrt(sf max_free G_i / m_i): omega_max^2 dt^2 <= 4 / sf, the reference's margin
        assert dt == pytest.approx(2.0 / np.sqrt(sf * max(rows[1] / 1.0, rows[2] / 0.5)))
    # a step already below the bound is kept
    _, _, dt = DynamicRelaxationAnalysis(dom, dt=0.01, mass="lumped").fictitious_mass(0.01, free, fixed)
    assert dt == 0.01
    # the reference's mass keeps the given step: m = sf dt^2 G / 4
    m, _, dt = DynamicRelaxationAnalysis(dom, safety_factor=1.1, dt=1.0).fictitious_mass(1.0, free, fixed)
    assert dt == 1.0 and np.allclose(m, 0.25 * 1.1 * rows)
    with pytest.raises(ValueError, match="mass must be"):
        DynamicRelaxationAnalysis(dom, mass="consistent")
