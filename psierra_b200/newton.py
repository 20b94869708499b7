"""Device-resident incremental Newton solver on the GPU assembly and PCG.

Everything that scales with the mesh stays on the device: one fused f_int + K_T
assembly per iteration (``GPUAssembler.assemble``), symmetric elimination of the
prescribed DOFs in place (``psx_csr_dirichlet``), the linear step by preconditioned CG
(``psx_pcg``, 3x3 block-Jacobi by default) and f_int-only evaluations for the line
search.  Only scalars (residual norms, solver status) reach the host.  The iteration
follows the reference's incremental Newton (psierra ``analysis/nonlinear_static.py:250-404``:
load ramp, test ||R_free|| < nr_tol * ||f_step_free||, backtracking line search with the
acceptance rules of ``analysis/line_search.py:120-260``).
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


@dataclass
class DeviceNewtonResult:
    u: torch.Tensor
    converged: bool
    steps_completed: int
    iteration_history: list[int] = field(default_factory=list)
    pcg_iterations: list[int] = field(default_factory=list)
    residual_history: list[float] = field(default_factory=list)
    step_lengths: list[float] = field(default_factory=list)  # accepted line-search alphas


class DeviceNewton:
    def __init__(self, asm: GPUAssembler, fixed_dofs, precision: str | None = None, pcg_tol: float = 1e-10,
                 pcg_maxiter: int = 20000, preconditioner: str = "block-jacobi") -> None:
        """``preconditioner``: "jacobi", "block-jacobi" or "two-level" (block-Jacobi plus
        the rigid-body modes of slices of the mesh, ``psierra_b200.coarse``)."""
        self.asm = asm
        self.precision = precision or asm.precision
        dev = asm.device
        n = 3 * asm.n_nodes
        self.n = n
        mask = np.zeros(n, dtype=np.uint8)
        mask[np.asarray(fixed_dofs, dtype=np.int64)] = 1
        self.fixed = torch.from_numpy(mask).to(dev)
        self.free = torch.from_numpy(mask == 0).to(dev)
        self.coarse = None
        if preconditioner == "two-level":
            from psierra_b200.coarse import CoarseSpace

            self.coarse = CoarseSpace(asm.X.view(-1, 3).cpu().numpy(), asm.pattern.conn, mask, device=dev)
            preconditioner = "block-jacobi"
        self.pcg = ConjugateGradientSolver(tolerance=pcg_tol, max_iterations=pcg_maxiter,
                                           preconditioner=preconditioner, device=dev)
        self.f = asm.new_f()
        self.k = asm.new_k(self.precision)
        self.ls = ContactAwareLineSearch()

    def tangent(self, u: torch.Tensor) -> torch.Tensor:
        """K_T(u) with prescribed rows/columns eliminated (CSR values on the device)."""
        self.asm.assemble(u, want_f=False, want_k=True, precision=self.precision, k_out=self.k)
        self._eliminate()
        return self.k

    def _eliminate(self) -> None:
        d = self.asm.dev
        vp = _lib.PSX_FP64 if self.k.dtype == torch.float64 else _lib.PSX_FP32_MIXED
        check(lib().psx_csr_dirichlet(self.n, ptr(d["indptr"]), ptr(d["indices"]), ptr(self.k), vp, ptr(self.fixed),
                                      torch.cuda.current_stream().cuda_stream), "psx_csr_dirichlet")

    def solve_linear(self, rhs: torch.Tensor) -> tuple[torch.Tensor, int]:
        """K x = rhs with the current eliminated tangent; rhs must be zero on fixed DOFs."""
        d = self.asm.dev
        x = torch.zeros_like(rhs)
        if self.coarse is not None:
            self.coarse.update(self.k, d["indptr"], d["indices"])
        res = self.pcg.solve_device(d["indptr"], d["indices"], self.k, rhs, x, nodal=True, coarse=self.coarse)
        if not res.converged:
            raise RuntimeError(f"Conjugate Gradient did not converge (info={res.iterations}).")
        return x, res.iterations

    def residual(self, u: torch.Tensor, f_step: torch.Tensor) -> tuple[torch.Tensor, float]:
        f, _ = self.asm.assemble(u, want_f=True, want_k=False, f_out=self.f)
        r = torch.where(self.free, f_step - f, torch.zeros_like(f))
        return r, float(torch.linalg.vector_norm(r))

    def solve(self, f_ext: torch.Tensor, u0: torch.Tensor | None = None, u_prescribed: torch.Tensor | None = None,
              n_steps: int = 10, nr_iterations: int = 25, nr_tol: float = 1e-8,
              polish: int = 0) -> DeviceNewtonResult:
        """Incremental Newton over ``n_steps`` load steps.

        ``polish`` extra full Newton steps follow convergence of the last load step,
        each kept only while it lowers the residual: an adjoint gradient is exact only
        at equilibrium, so its callers converge to the round-off floor rather than to
        ``nr_tol``.
        """
        n = self.n
        u = torch.zeros(n, dtype=torch.float64, device=self.asm.device) if u0 is None else u0.clone()
        up = torch.zeros_like(u) if u_prescribed is None else u_prescribed
        hist, pcg_its, rhist, alphas = [], [], [], []
        for step in range(1, n_steps + 1):
            lam = step / n_steps
            u_acc = u.clone()
            u = torch.where(self.free, u, lam * up)
            f_step = lam * f_ext
            fnorm = float(torch.linalg.vector_norm(torch.where(self.free, f_step, torch.zeros_like(f_step))))
            # analysis/nonlinear_static.py:275-331: the step's force scale, or (no load) the
            # first iteration's max(||R||, ||f_int,free||, 1), kept for the whole step
            ref = fnorm if fnorm >= 1e-12 else None
            converged = False
            it = 0
            for it in range(1, nr_iterations + 1):
                f, _ = self.asm.assemble(u, want_f=True, want_k=True, precision=self.precision, f_out=self.f,
                                         k_out=self.k)
                self._eliminate()
                r = torch.where(self.free, f_step - f, torch.zeros_like(f))
                rn = float(torch.linalg.vector_norm(r))
                rhist.append(rn)
                if ref is None:
                    fi = float(torch.linalg.vector_norm(torch.where(self.free, f, torch.zeros_like(f))))
                    ref = max(rn, fi, 1.0)
                tol = nr_tol * ref
                if not np.isfinite(rn):
                    break
                if rn < tol:
                    converged = True
                    break
                du, its = self.solve_linear(r)
                pcg_its.append(its)

                def trial(alpha, du=du, u=u, f_step=f_step):
                    _, cn = self.residual(u + alpha * du, f_step)
                    return cn

                res = self.ls.search(trial, rn, tol, contact_active=False, reference_norm=ref)
                if not res.success:
                    break
                u = u + res.alpha * du
                alphas.append(float(res.alpha))
            if not converged:
                return DeviceNewtonResult(u_acc, False, step - 1, hist, pcg_its, rhist, alphas)
            hist.append(it)
        u = self._polish(u, f_step, rhist[-1], polish, pcg_its, rhist)
        return DeviceNewtonResult(u, True, n_steps, hist, pcg_its, rhist, alphas)

    def _polish(self, u, f_step, rn, n_extra, pcg_its, rhist):
        for _ in range(n_extra):
            if rn == 0.0:
                break
            self.asm.assemble(u, want_f=False, want_k=True, precision=self.precision, k_out=self.k)
            self._eliminate()
            r, _ = self.residual(u, f_step)
            du, its = self.solve_linear(r)
            pcg_its.append(its)
            u_new = u + du
            _, rn_new = self.residual(u_new, f_step)
            if not rn_new < rn:
                break
            u, rn = u_new, rn_new
            rhist.append(rn)
        return u
