"""Host drivers that call the GPU elements through the domain: Newton and dynamic relaxation.

These restate the no-contact path of pSierra's drivers so that they run where the
reference is not installed; with the reference present, its own drivers call the same
GPU elements through ``SolidDomain`` unchanged.

* ``NonlinearStaticAnalysis.solve`` -- incremental Newton-Raphson with prescribed-DOF
  ramping, the residual test ``||R_free|| < nr_tol * f_ref`` and backtracking line search
  (psierra ``analysis/nonlinear_static.py:73-549``, no contact so the augmentation loop
  runs once).  State rollback and the returned reactions follow the reference.
* ``ContactAwareLineSearch`` -- the acceptance rules of ``analysis/line_search.py:68-260``
  (direct convergence, strict decrease, Armijo with c1 = 2e-4, post-loop fallback on the
  best finite trial; inverted trials are halved).
* ``DynamicRelaxationAnalysis.solve`` -- explicit pseudo-dynamics with the Gerschgorin
  fictitious mass and kinetic or viscous damping (``analysis/dynamic_relaxation.py:32-468``).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from psierra_b200.domain import DirichletManager
from psierra_b200.solver import DirectSolver


def is_element_inversion_error(exc: BaseException) -> bool:
    """Classifier of ``analysis/line_search.py:10-33``."""
    if isinstance(exc, FloatingPointError):
        return True
    if isinstance(exc, ValueError):
        msg = str(exc).lower()
        keys = ("element inversion", "negative jacobian", "det(f)", "outside admissible", "admissible range",
                "zero surface area", "degenerate")
        return any(k in msg for k in keys)
    return False


@dataclass(frozen=True)
class LineSearchResult:
    success: bool
    alpha: float
    candidate_norm: float
    iterations: int
    element_inversion_encountered: bool
    accepted_as_contact_fallback: bool
    rejection_reason: str | None = None


class ContactAwareLineSearch:
    def __init__(self, max_iterations: int = 16, contraction_factor: float = 0.5, armijo_c1: float = 2.0e-4,
                 full_step_tolerance: float = 1.5, contact_fallback_tolerance: float = 5.0) -> None:
        if max_iterations < 1:
            raise ValueError("max_iterations must be at least 1")
        if not 0.0 < contraction_factor < 1.0:
            raise ValueError("contraction_factor must be in (0, 1)")
        if not 0.0 < armijo_c1 < 0.5:
            raise ValueError("armijo_c1 must be in (0, 0.5)")
        self.max_iterations = int(max_iterations)
        self.contraction_factor = float(contraction_factor)
        self.armijo_c1 = float(armijo_c1)
        self.full_step_tolerance = float(full_step_tolerance)
        self.contact_fallback_tolerance = float(contact_fallback_tolerance)

    def search(self, eval_fn, current_norm: float, inner_tolerance: float, *, contact_active: bool = False,
               reference_norm: float | None = None) -> LineSearchResult:
        alpha, best_norm, best_alpha = 1.0, np.inf, 1.0
        inverted_any = False
        scale = max(current_norm, reference_norm) if reference_norm is not None else current_norm
        for it in range(1, self.max_iterations + 1):
            try:
                cand = float(eval_fn(alpha))
                inverted = False
            except Exception as exc:  # noqa: BLE001 - classified below, others re-raised
                if not is_element_inversion_error(exc):
                    raise
                inverted, cand = True, np.inf
            if inverted or not np.isfinite(cand):
                inverted_any = True
                alpha *= self.contraction_factor
                continue
            if cand < best_norm:
                best_norm, best_alpha = cand, alpha
            accept = (cand <= inner_tolerance or cand <= current_norm
                      or cand ** 2 <= (1.0 - 2.0 * self.armijo_c1 * alpha) * current_norm ** 2
                      or (contact_active and it == 1 and alpha == 1.0 and cand < self.full_step_tolerance * scale))
            if accept:
                return LineSearchResult(True, alpha, cand, it, inverted_any, False)
            alpha *= self.contraction_factor
        if np.isfinite(best_norm) and best_norm < self.contact_fallback_tolerance * scale and \
                (contact_active or not inverted_any):
            return LineSearchResult(True, best_alpha, best_norm, self.max_iterations, inverted_any, True)
        reason = ("Element inversion detected across all evaluated step lengths"
                  if (not np.isfinite(best_norm) and inverted_any)
                  else f"Residual {best_norm:.4e} exceeded fallback tolerance "
                       f"{self.contact_fallback_tolerance * scale:.4e}")
        return LineSearchResult(False, best_alpha, best_norm, self.max_iterations, inverted_any, False, reason)


@dataclass
class NonlinearStaticResult:
    displacement: np.ndarray
    reactions: np.ndarray
    converged: bool
    steps_completed: int
    iteration_history: list[int] = field(default_factory=list)


def _manager(dirichlet, n_dofs: int):
    if isinstance(dirichlet, list):
        mgr = DirichletManager(n_dofs)
        for c in dirichlet:
            mgr.add_constraint(c)
        return mgr
    return dirichlet


class NonlinearStaticAnalysis:
    def __init__(self, domain, linear_solver=None) -> None:
        self.domain = domain
        self.linear_solver = linear_solver if linear_solver is not None else DirectSolver()

    def solve(self, dirichlet, f_ext=None, n_steps: int = 10, nr_iterations: int = 25, nr_tol: float = 1e-4,
              verbose: bool = False, line_search: ContactAwareLineSearch | None = None) -> NonlinearStaticResult:
        dom = self.domain
        n = dom.n_dofs
        f_ext = np.zeros(n) if f_ext is None else np.asarray(f_ext, dtype=np.float64)
        if f_ext.shape != (n,) or not np.all(np.isfinite(f_ext)):
            raise ValueError("f_ext must be a finite vector of shape (n_dofs,)")
        ls = line_search if line_search is not None else ContactAwareLineSearch()
        mgr = _manager(dirichlet(1, n_steps) if callable(dirichlet) else dirichlet, n)
        free, p_dofs, u_p = mgr.free_dofs, mgr.prescribed_dofs, mgr.prescribed_values
        if len(free) == 0:
            raise ValueError("All degrees of freedom are constrained. Nothing to solve.")
        u_current = dom.u.copy()
        history: list[int] = []
        for step in range(1, n_steps + 1):
            lam = step / n_steps
            acc_u, acc_v, acc_a = dom.u.copy(), dom.v.copy(), dom.a.copy()
            if callable(dirichlet):
                mgr = _manager(dirichlet(step, n_steps), n)
                free, p_dofs, u_p = mgr.free_dofs, mgr.prescribed_dofs, mgr.prescribed_values
                u_current[p_dofs] = u_p
            elif len(p_dofs) > 0:
                u_current[p_dofs] = lam * u_p
            f_step_free = (lam * f_ext)[free]
            fnorm = float(np.linalg.norm(f_step_free))
            f_ref = fnorm if fnorm >= 1e-12 else None
            converged = False
            iteration = 0
            for iteration in range(1, nr_iterations + 1):
                dom.update_state(u=u_current)
                try:
                    f_int = dom.assemble_internal_forces()
                    K_tan = dom.assemble_tangent_stiffness_matrix()
                except (ValueError, FloatingPointError):
                    dom.update_state(u=acc_u, v=acc_v, a=acc_a)
                    raise
                r_free = f_step_free - f_int[free]
                rnorm = float(np.linalg.norm(r_free))
                if not np.isfinite(rnorm):
                    break
                if f_ref is None:
                    f_ref = max(rnorm, float(np.linalg.norm(f_int[free])), 1.0)
                tol = nr_tol * f_ref
                if verbose:
                    print(f"  step {step} iter {iteration}: |R| = {rnorm:.4e} rel = {rnorm / f_ref:.4e}")
                if rnorm < tol:
                    converged = True
                    break
                K_free = K_tan[free, :][:, free].tocsc()
                try:
                    du = self.linear_solver.solve(K_free, r_free)
                except (RuntimeError, np.linalg.LinAlgError):
                    break
                if not np.all(np.isfinite(du)):
                    break

                def trial(alpha, du=du):
                    u_cand = u_current.copy()
                    u_cand[free] += alpha * du
                    if not np.all(np.isfinite(u_cand)):
                        return np.inf
                    dom.update_state(u=u_cand)
                    return float(np.linalg.norm(f_step_free - dom.assemble_internal_forces()[free]))

                res = ls.search(trial, rnorm, tol, contact_active=False, reference_norm=f_ref)
                if not res.success:
                    break
                u_current[free] += res.alpha * du
            if not converged:
                u_current = acc_u
                dom.update_state(u=acc_u, v=acc_v, a=acc_a)
                reactions = dom.assemble_internal_forces() - ((step - 1) / n_steps) * f_ext
                return NonlinearStaticResult(u_current, reactions, False, step - 1, history)
            history.append(iteration)
            dom.commit_state()
        dom.update_state(u=u_current)
        reactions = dom.assemble_internal_forces() - f_ext
        return NonlinearStaticResult(u_current, reactions, True, n_steps, history)


@dataclass
class DynamicRelaxationResult:
    displacement: np.ndarray
    reactions: np.ndarray
    converged: bool
    steps_completed: int
    residual_norm: float
    relative_residual: float
    kinetic_energy: float
    kinetic_peaks: int
    residual_history: list[float] = field(default_factory=list)


class DynamicRelaxationAnalysis:
    def __init__(self, domain, damping_type: str = "kinetic", safety_factor: float = 1.1,
                 viscous_damping: float | None = None, dt: float = 1.0, mass: str = "gerschgorin") -> None:
        """``mass``: "gerschgorin" (the reference's fictitious mass) or "lumped" (the row
        sums of the domain's consistent mass matrix; see ``fictitious_mass``)."""
        self.domain = domain
        self.damping_type = damping_type.lower()
        if self.damping_type not in ("kinetic", "viscous"):
            raise ValueError(f"damping_type must be 'kinetic' or 'viscous', got '{damping_type}'")
        self.mass = mass.lower()
        if self.mass not in ("gerschgorin", "lumped"):
            raise ValueError(f"mass must be 'gerschgorin' or 'lumped', got '{mass}'")
        self.safety_factor = float(safety_factor)
        self.viscous_damping = viscous_damping
        self.dt = float(dt)

    def fictitious_mass(self, dt: float, free, p_dofs):
        """(diagonal mass, its inverse on the free DOFs, pseudo-time step).

        "gerschgorin", the reference's (``dynamic_relaxation.py:87-128``, no contact):
        m_i = sf dt^2 G_i / 4, with G_i the absolute row sum of the small-strain
        stiffness, so that every mode is stable at the given dt.  "lumped" (a build
        option; the reference has none): m_i = the row sum of the consistent mass matrix
        (rho times volume per node), and the step becomes 2 / sqrt(sf max_i G_i / m_i)
        over the free DOFs when dt is larger, the same stability margin."""
        K0 = self.domain.assemble_stiffness_matrix()
        rows = np.asarray(np.abs(K0).sum(axis=1)).ravel()
        mx = float(rows.max()) if rows.size and rows.max() > 0 else 1.0
        rows = np.maximum(rows, 1e-6 * mx)
        if self.mass == "lumped":
            m = np.asarray(self.domain.assemble_mass_matrix().sum(axis=1), dtype=np.float64).ravel()
            if not np.all(m[free] > 0.0):
                raise ValueError("the lumped mass has a non-positive entry on a free DOF")
            dt = min(dt, 2.0 / np.sqrt(self.safety_factor * float(np.max(rows[free] / m[free]))))
        else:
            m = 0.25 * self.safety_factor * dt ** 2 * rows
        inv = np.zeros_like(m)
        inv[free] = 1.0 / m[free]
        inv[p_dofs] = 0.0
        return m, inv, dt

    def solve(self, dirichlet, f_ext=None, tol: float = 1e-5, max_steps: int = 5000, min_steps: int = 10,
              verbose: bool = False) -> DynamicRelaxationResult:
        dom = self.domain
        n = dom.n_dofs
        mgr = _manager(dirichlet, n)
        free, p_dofs, u_p = mgr.free_dofs, mgr.prescribed_dofs, mgr.prescribed_values
        if len(free) == 0:
            raise ValueError("All degrees of freedom are constrained. Nothing to solve.")
        f = np.zeros(n) if f_ext is None else np.asarray(f_ext, dtype=np.float64).ravel()
        ref = float(np.linalg.norm(f[free]))
        ref = 1.0 if ref < 1e-12 else ref
        m_diag, inv_m, dt = self.fictitious_mass(self.dt, free, p_dofs)
        u = dom.u.copy()
        u[p_dofs] = u_p
        v = np.zeros(n)
        dom.update_state(u=u, v=v)
        f_int = dom.assemble_internal_forces()
        r = f - f_int
        a = inv_m * r
        a[p_dofs] = 0.0
        res = float(np.linalg.norm(r[free]))
        rel = res / ref
        if self.damping_type == "kinetic":
            v_half = 0.5 * dt * a
        else:
            c = self.viscous_damping if self.viscous_damping is not None else 0.4
            c1, c2 = (2.0 - c * dt) / (2.0 + c * dt), (2.0 * dt) / (2.0 + c * dt)
            v_half = 0.5 * c2 * a
        v_half[p_dofs] = 0.0
        prev_ek, peaks, hist, converged, step, ek = 0.0, 0, [res], False, 0, 0.0
        for step in range(1, max_steps + 1):
            u_prev, a_prev = u.copy(), a.copy()
            u = u + dt * v_half
            u[p_dofs] = u_p
            dom.update_state(u=u, v=v_half)
            try:
                f_int = dom.assemble_internal_forces()
            except (ValueError, FloatingPointError):
                u = 0.5 * (u + u_prev)
                dom.update_state(u=u, v=np.zeros(n))
                f_int = dom.assemble_internal_forces()
            r = f - f_int
            a = inv_m * r
            a[p_dofs] = 0.0
            res = float(np.linalg.norm(r[free]))
            rel = res / ref
            hist.append(res)
            if self.damping_type == "kinetic":
                v_next = v_half + dt * a
                v_next[p_dofs] = 0.0
                v_mid = 0.5 * (v_half + v_next)
                ek = 0.5 * float(np.sum(m_diag[free] * v_mid[free] ** 2))
                if step > 1 and ek < prev_ek:
                    peaks += 1
                    u_peak = u - 1.5 * dt * v_half + 0.5 * dt ** 2 * a_prev
                    u_peak[p_dofs] = u_p
                    try:
                        dom.update_state(u=u_peak, v=np.zeros(n))
                        f_test = dom.assemble_internal_forces()
                        if np.all(np.isfinite(f_test)):
                            u, f_int = u_peak, f_test
                    except (ValueError, FloatingPointError):
                        u = u_prev
                        dom.update_state(u=u, v=np.zeros(n))
                        f_int = dom.assemble_internal_forces()
                    r = f - f_int
                    a = inv_m * r
                    a[p_dofs] = 0.0
                    res = float(np.linalg.norm(r[free]))
                    rel = res / ref
                    v_next = 0.5 * dt * a
                    v_next[p_dofs] = 0.0
                    prev_ek = 0.0
                else:
                    prev_ek = ek
                v_half = v_next
            else:
                v_half = c1 * v_half + c2 * a
                v_half[p_dofs] = 0.0
                ek = 0.5 * float(np.sum(m_diag[free] * v_half[free] ** 2))
            if verbose and (step == 1 or step % 50 == 0):
                print(f"  DR step {step}: |R| = {res:.4e} rel = {rel:.4e}")
            if step >= min_steps and rel <= tol:
                converged = True
                break
        dom.update_state(u=u, v=np.zeros(n), a=np.zeros(n))
        return DynamicRelaxationResult(u.copy(), f_int - f, converged, step, res, rel, ek, peaks, hist)
