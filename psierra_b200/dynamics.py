"""Device-resident implicit dynamics (generalized-alpha) on the GPU assembly.

Restates ``NonlinearDynamicAnalysis.solve`` (psierra ``analysis/nonlinear_dynamic.py``)
for the path without contact and with fixed time steps:

* constants of Chung & Hulbert from the spectral radius rho_inf (``:110-117``) and the
  Newmark coefficients a0..a5 (``:349-356, 458-465``);
* constant consistent mass M and small-strain stiffness K_0, Rayleigh damping
  ``C = alpha_R M + beta_R K_0`` (``:370-378``, ``damping/rayleigh.py:21-26``);
* initial acceleration from ``M_ff a0 = f_ext - C v - f_int(u0)`` (``:388-409``);
* per step, Newton on the midpoint residual
  ``R = f_ext - M a_mid - C v_mid - f_int(u_mid)`` (``:560-622``) with the effective
  tangent ``(1 - alpha_f) K_T(u_mid) + (1 - alpha_m) a0 M + (1 - alpha_f) a1 C``
  (``:640-644``), the same line search (``:658-712``) and the Newmark update of v and a
  after convergence.

Everything stays on the device: the effective tangent comes from one fused sweep
(``psx_tet4_assemble_effective``), M a and K_0 v from ``psx_csr_spmv``, the linear
steps from block-Jacobi PCG on the eliminated tangent; only residual norms reach the host.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import torch

from psierra_b200 import _lib
from psierra_b200._lib import check, lib, ptr
from psierra_b200.analysis import ContactAwareLineSearch
from psierra_b200.assembler import GPUAssembler
from psierra_b200.solver import ConjugateGradientSolver


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


@dataclass
class DeviceDynamicResult:
    u: torch.Tensor
    v: torch.Tensor
    a: torch.Tensor
    converged: bool
    steps_completed: int
    iteration_history: list[int] = field(default_factory=list)
    pcg_iterations: list[int] = field(default_factory=list)


class DeviceGeneralizedAlpha:
    def __init__(self, asm: GPUAssembler, fixed_dofs, damping=(0.0, 0.0), spectral_radius: float = 0.8,
                 precision: str | None = None, pcg_tol: float = 1e-12, pcg_maxiter: int = 20000,
                 preconditioner: str = "block-jacobi"):
        if not (0.0 <= spectral_radius <= 1.0):
            raise ValueError(f"spectral_radius must be in [0.0, 1.0], got {spectral_radius}")
        rho = float(spectral_radius)
        self.alpha_m = (2.0 * rho - 1.0) / (rho + 1.0)
        self.alpha_f = rho / (rho + 1.0)
        self.gamma = 0.5 - self.alpha_m + self.alpha_f
        self.beta = 0.25 * (1.0 - self.alpha_m + self.alpha_f) ** 2
        self.alpha_r, self.beta_r = (float(x) for x in damping)
        self.asm = asm
        self.precision = precision or asm.precision
        dev = asm.device
        n = 3 * asm.n_nodes
        self.n = n
        mask = np.zeros(n, dtype=np.uint8)
        mask[np.asarray(fixed_dofs, dtype=np.int64)] = 1
        self.fixed = torch.from_numpy(mask).to(dev)
        self.free = torch.from_numpy(mask == 0).to(dev)
        _, self.M = asm.assemble(None, mass=True, precision="fp64")
        _, self.K0 = asm.assemble(None, linear=True, precision="fp64")
        self.M = self.M.clone()
        self.K0 = self.K0.clone()
        self.pcg = ConjugateGradientSolver(tolerance=pcg_tol, max_iterations=pcg_maxiter,
                                           preconditioner=preconditioner, device=dev)
        self.k = asm.new_k(self.precision)
        self.f = asm.new_f()
        self.ls = ContactAwareLineSearch()

    # ------------------------------------------------------------------ helpers
    def _spmv(self, vals: torch.Tensor, x: torch.Tensor, alpha: float, beta: float, y: torch.Tensor) -> torch.Tensor:
        d = self.asm.dev
        vp = _lib.PSX_FP64 if vals.dtype == torch.float64 else _lib.PSX_FP32_MIXED
        check(lib().psx_csr_spmv(self.n, ptr(d["indptr"]), ptr(d["indices"]), ptr(vals), vp, ptr(x), alpha, beta,
                                 ptr(y), _stream()), "psx_csr_spmv")
        return y

    def _inertia_damping(self, a_mid: torch.Tensor, v_mid: torch.Tensor) -> torch.Tensor:
        """M a_mid + C v_mid = M (a_mid + alpha_R v_mid) + beta_R K_0 v_mid."""
        y = torch.empty_like(a_mid)
        self._spmv(self.M, a_mid + self.alpha_r * v_mid, 1.0, 0.0, y)
        if self.beta_r != 0.0:
            self._spmv(self.K0, v_mid, self.beta_r, 1.0, y)
        return y

    def _eliminate(self, vals: torch.Tensor) -> None:
        d = self.asm.dev
        vp = _lib.PSX_FP64 if vals.dtype == torch.float64 else _lib.PSX_FP32_MIXED
        check(lib().psx_csr_dirichlet(self.n, ptr(d["indptr"]), ptr(d["indices"]), ptr(vals), vp, ptr(self.fixed),
                                      _stream()), "psx_csr_dirichlet")

    def _solve(self, vals: torch.Tensor, rhs: torch.Tensor) -> tuple[torch.Tensor, int]:
        d = self.asm.dev
        x = torch.zeros_like(rhs)
        res = self.pcg.solve_device(d["indptr"], d["indices"], vals, rhs, x, nodal=True)
        if not res.converged:
            raise RuntimeError(f"Conjugate Gradient did not converge (info={res.iterations}).")
        return x, res.iterations

    def _masked(self, x: torch.Tensor) -> torch.Tensor:
        return torch.where(self.free, x, torch.zeros_like(x))

    # ------------------------------------------------------------------ driver
    def solve(self, f_ext: torch.Tensor, dt: float, n_steps: int, nr_iterations: int = 15, nr_tol: float = 1e-4,
              u0: torch.Tensor | None = None, v0: torch.Tensor | None = None) -> DeviceDynamicResult:
        asm = self.asm
        dev = asm.device
        am, af, g, b = self.alpha_m, self.alpha_f, self.gamma, self.beta
        a0 = 1.0 / (b * dt ** 2)
        a1 = g / (b * dt)
        a2 = 1.0 / (b * dt)
        a3 = 1.0 / (2.0 * b) - 1.0
        a4 = g / b - 1.0
        a5 = dt * 0.5 * (g / b - 2.0)
        f_ext = f_ext.to(dev, torch.float64)
        u = torch.zeros(self.n, dtype=torch.float64, device=dev) if u0 is None else self._masked(u0.clone())
        v = torch.zeros_like(u) if v0 is None else self._masked(v0.clone())
        fn = float(torch.linalg.vector_norm(self._masked(f_ext)))
        f_ref = fn if fn >= 1e-12 else 1.0
        tol = nr_tol * f_ref
        # initial acceleration: M_ff a = f_ext - C v - f_int(u)
        f0, _ = asm.assemble(u, want_f=True, want_k=False, f_out=self.f)
        Cv = self._inertia_damping(torch.zeros_like(v), v)
        r0 = self._masked(f_ext - Cv - f0)
        Mel = self.M.clone()
        self._eliminate(Mel)
        acc, _ = self._solve(Mel, r0)
        c_t = 1.0 - af
        c_m = (1.0 - am) * a0 + (1.0 - af) * a1 * self.alpha_r
        c_0 = (1.0 - af) * a1 * self.beta_r
        hist, pcg_its = [], []

        def state(u_i):
            a_i = a0 * (u_i - u) - a2 * v - a3 * acc
            v_i = a1 * (u_i - u) - a4 * v - a5 * acc
            return ((1.0 - af) * u_i + af * u, (1.0 - af) * v_i + af * v, (1.0 - am) * a_i + am * acc)

        def residual(u_i):
            u_mid, v_mid, a_mid = state(u_i)
            f, _ = asm.assemble(u_mid, want_f=True, want_k=False, f_out=self.f)
            r = self._masked(f_ext - self._inertia_damping(a_mid, v_mid) - f)
            return r, float(torch.linalg.vector_norm(r))

        for step in range(1, n_steps + 1):
            u_i = u.clone()
            converged = False
            it = 0
            for it in range(1, nr_iterations + 1):
                u_mid, v_mid, a_mid = state(u_i)
                f, _ = asm.assemble_effective(u_mid, c_t, c_m, c_0, want_f=True, precision=self.precision,
                                              f_out=self.f, k_out=self.k)
                r = self._masked(f_ext - self._inertia_damping(a_mid, v_mid) - f)
                rn = float(torch.linalg.vector_norm(r))
                if not np.isfinite(rn):
                    break
                if rn < tol:
                    converged = True
                    break
                self._eliminate(self.k)
                du, its = self._solve(self.k, r)
                pcg_its.append(its)

                def trial(alpha, du=du, u_i=u_i):
                    return residual(u_i + alpha * du)[1]

                res = self.ls.search(trial, rn, tol, contact_active=False, reference_norm=f_ref)
                if not res.success:
                    break
                u_i = u_i + res.alpha * du
            if not converged:
                return DeviceDynamicResult(u, v, acc, False, step - 1, hist, pcg_its)
            a_new = a0 * (u_i - u) - a2 * v - a3 * acc
            v_new = a1 * (u_i - u) - a4 * v - a5 * acc
            u, v, acc = u_i, v_new, a_new
            hist.append(it - 1)  # Newton updates taken, as the reference records them (:721)
        return DeviceDynamicResult(u, v, acc, True, n_steps, hist, pcg_its)
