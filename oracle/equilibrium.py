"""Static equilibrium of the reference forward model, and the gradients it implies.

Test infrastructure only: the checker of the adjoint path.  ``solve_static`` is the
reference's incremental Newton iteration without contact and with full steps
(psierra ``analysis/nonlinear_static.py:290-404``: assemble f_int and K_T, the residual
R = f_ext,step - f_int on the free DOFs, ``DirectSolver`` = SuperLU on the free-DOF
block, ``solver/sparse_linear_solver.py:10-19``), on the oracle's element sweep and
COO->CSR assembly with one NeoHookean per element (``oracle.assembly``).  It iterates
to a tight residual so that central differences of its solution have a rounding floor
far below the 1e-5 bar they check.

``force_parameter_gradients`` restates the exact parameter derivative of the element
force: S and the tangent are linear in (mu, kappa) at fixed F
(``material/neohookean.py:87-114``), so d f_e / d mu_e = f_e(mu=1, kappa=0) and
d f_e / d kappa_e = f_e(mu=0, kappa=1).
"""
from __future__ import annotations

import numpy as np
import scipy.sparse.linalg as spla

from oracle import vectorized
from oracle.assembly import assemble_sparse, assemble_vector, coo_indices, element_dofs


def assemble(nodes, elements, u, mu, kappa):
    """(f_int (n,), K_T CSR) of the reference assembly at nodal displacements u (N, 3)."""
    k, f = vectorized.element_force_and_tangent(nodes, elements, u, mu, kappa)
    ed = element_dofs(elements)
    r, c = coo_indices(ed)
    n = 3 * nodes.shape[0]
    return assemble_vector(f, ed, n), assemble_sparse(k, r, c, n)


def solve_static(nodes, elements, mu, kappa, fixed_dofs, f_ext, n_steps: int = 2, rtol: float = 1e-14,
                 max_iterations: int = 30) -> np.ndarray:
    """u (3N,) with f_int(u) = f_ext on the free DOFs (u = 0 on ``fixed_dofs``).

    ``n_steps`` load increments f_ext * step / n_steps, full Newton steps with the direct
    solver, each increment iterated until ||R_free|| <= rtol ||f_ext,step,free|| or until
    the residual stops falling (the rounding floor)."""
    n = 3 * nodes.shape[0]
    free = np.setdiff1d(np.arange(n), np.asarray(fixed_dofs))
    u = np.zeros(n)
    for step in range(1, n_steps + 1):
        f_step = f_ext * (step / n_steps)
        ref = np.linalg.norm(f_step[free])
        best = np.inf
        for _ in range(max_iterations):
            f_int, K = assemble(nodes, elements, u.reshape(-1, 3), mu, kappa)
            r = f_step[free] - f_int[free]
            rn = np.linalg.norm(r)
            if rn <= rtol * ref or rn >= best:
                break
            best = rn
            Kff = K[free][:, free].tocsc()
            u[free] += spla.spsolve(Kff, r)
        else:
            raise RuntimeError("oracle Newton did not converge")
    return u


def force_parameter_gradients(nodes, elements, u, w):
    """(w . d f / d mu_e, w . d f / d kappa_e), each (E,), for a cotangent w (3N,)."""
    el = np.asarray(elements, dtype=np.int64)
    E = el.shape[0]
    ed = element_dofs(el)
    wl = np.asarray(w)[ed]  # (E, d)
    _, f_mu = vectorized.element_force_and_tangent(nodes, el, u, np.ones(E), np.zeros(E))
    _, f_ka = vectorized.element_force_and_tangent(nodes, el, u, np.zeros(E), np.ones(E))
    return np.einsum("ed,ed->e", wl, f_mu), np.einsum("ed,ed->e", wl, f_ka)
