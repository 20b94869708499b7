"""The oracle's equilibrium solve and parameter derivatives (CPU), pinned to the reference.

* ``solve_static`` reproduces the reference's own converged Newton solution of the
  10 x 2 x 2 cantilever (``tests/golden/newton_beam.npz``, written by running
  ``NonlinearStaticAnalysis`` with ``DirectSolver``) to its Newton tolerance.
* ``force_parameter_gradients`` follows from the linearity of the NeoHookean stress in
  (mu, kappa) at fixed F: f_e(mu, kappa) = mu f_e(1, 0) + kappa f_e(0, 1), checked
  with the reference-restating element on random moduli and a deformed state.
"""
from __future__ import annotations

import numpy as np

from conftest import golden, rel_2
from oracle import equilibrium, vectorized
from oracle.assembly import element_dofs
from psierra_b200 import meshgen


def test_solve_static_reproduces_reference_newton_beam():
    g = golden("newton_beam")
    m = meshgen.box_tet4(1.0, 0.1, 0.1, 10, 2, 2)
    fixed = np.concatenate([3 * g["clamp"] + c for c in range(3)])
    u = equilibrium.solve_static(m.nodes, m.elements, float(g["mu"]), float(g["kappa"]), fixed, g["f_ext"],
                                 n_steps=4)
    assert rel_2(u, g["u"]) < 1e-12  # observed 1.6e-14
    # the residual's rounding floor: element forces of order mu cancel to the small load
    # (the reference's own solution sits at 7.9e-11 of ||f_ext|| on the same assembly)
    f_int, _ = equilibrium.assemble(m.nodes, m.elements, u.reshape(-1, 3), float(g["mu"]), float(g["kappa"]))
    free = np.setdiff1d(np.arange(m.n_dofs), fixed)
    assert np.linalg.norm(f_int[free] - g["f_ext"][free]) < 1e-9 * np.linalg.norm(g["f_ext"][free])


def test_parameter_gradients_follow_from_linearity():
    m = meshgen.box_tet4(1.0, 0.4, 0.3, 3, 2, 2)
    rng = np.random.default_rng(2)
    u = 0.03 * rng.normal(size=(m.n_nodes, 3))
    mu = rng.uniform(500.0, 2000.0, m.n_elements)
    kappa = 50.0 * mu * rng.uniform(0.5, 1.5, m.n_elements)
    w = rng.normal(size=m.n_dofs)
    gmu, gka = equilibrium.force_parameter_gradients(m.nodes, m.elements, u, w)
    _, f = vectorized.element_force_and_tangent(m.nodes, m.elements, u, mu, kappa)
    wl = w[element_dofs(m.elements)]
    direct = np.einsum("ed,ed->e", wl, f)
    assert np.abs(mu * gmu + kappa * gka - direct).max() <= 1e-12 * np.abs(direct).max()
    # and central differences of w.f in mu_e of one element
    e, h = 7, 1e-3 * mu[7]
    mp, mm = mu.copy(), mu.copy()
    mp[e] += h
    mm[e] -= h
    fp = vectorized.element_force_and_tangent(m.nodes, m.elements[e:e + 1], u, mp[e:e + 1], kappa[e:e + 1])[1]
    fm = vectorized.element_force_and_tangent(m.nodes, m.elements[e:e + 1], u, mm[e:e + 1], kappa[e:e + 1])[1]
    fd = float(wl[e] @ (fp[0] - fm[0])) / (2 * h)
    assert abs(fd - gmu[e]) <= 1e-9 * abs(gmu[e])
