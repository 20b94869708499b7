"""Differentiation of the internal force and of the static equilibrium (torch.autograd).

pSierra is gradient-free: ``MaterialParameterIdentifier`` drives scipy least squares
with finite-difference Jacobians of a full forward solve per parameter
(psierra ``inverse/parameter_identification.py:259-416``).  Here the gradient comes
from a hand-written adjoint kernel (``psx_tet4_adjoint``):

* ``InternalForce`` -- ``f_int(X, u, mu_e, kappa_e)`` with backward
  ``(w^T df/dX, K_T(u) w, w^T df/dmu_e, w^T df/dkappa_e)``; F is recomputed from (X, u)
  in the backward pass, nothing per element is stored.
* ``StaticEquilibrium`` -- ``u*(mu_e, kappa_e, f_ext)`` solving f_int(u*) = f_ext on the
  free DOFs with the device Newton solver; backward solves the adjoint system
  ``K_T(u*) lam = dL/du`` with the same PCG (K_T is symmetric) and returns
  ``-lam^T df/dmu_e``, ``-lam^T df/dkappa_e`` and ``lam`` for f_ext.
* ``identify_shear_moduli`` -- per-element shear-modulus identification from surface
  displacements (bulk modulus tied to the shear modulus by a fixed ratio), by L-BFGS-B
  on those gradients.
"""
from __future__ import annotations

import numpy as np
import torch

from psierra_b200.assembler import GPUAssembler
from psierra_b200.newton import DeviceNewton


def _set_params(asm: GPUAssembler, X, mu_e, kappa_e) -> None:
    if X is not None:
        asm.X.copy_(X.detach().reshape(asm.X.shape))
    asm.mu_e = mu_e.detach().contiguous()
    asm.kappa_e = kappa_e.detach().contiguous()


class InternalForce(torch.autograd.Function):
    @staticmethod
    def forward(ctx, X, u, mu_e, kappa_e, asm: GPUAssembler):
        _set_params(asm, X, mu_e, kappa_e)
        f, _ = asm.assemble(u.detach().reshape(-1).contiguous(), want_f=True, want_k=False, precision="fp64")
        ctx.asm = asm
        ctx.save_for_backward(X, u, mu_e, kappa_e)
        return f.clone()

    @staticmethod
    def backward(ctx, gf):
        X, u, mu_e, kappa_e = ctx.saved_tensors
        asm = ctx.asm
        _set_params(asm, X, mu_e, kappa_e)
        w = gf.detach().reshape(-1).contiguous()
        ud = u.detach().reshape(-1).contiguous()
        gX, gmu, gk = asm.adjoint(ud, w)
        gu = asm.kv(ud, w, precision="fp64")
        return gX.reshape(X.shape), gu.reshape(u.shape), gmu, gk, None


def internal_force(asm: GPUAssembler, X, u, mu_e, kappa_e):
    return InternalForce.apply(X, u, mu_e, kappa_e, asm)


class StaticEquilibrium(torch.autograd.Function):
    @staticmethod
    def forward(ctx, mu_e, kappa_e, f_ext, newton: DeviceNewton, n_steps: int, nr_tol: float, polish: int, u0=None):
        asm = newton.asm
        _set_params(asm, None, mu_e, kappa_e)
        res = newton.solve(f_ext.detach(), u0=None if u0 is None else u0.detach(), n_steps=n_steps, nr_tol=nr_tol,
                           polish=polish)
        if not res.converged:
            raise RuntimeError("static equilibrium did not converge")
        ctx.newton = newton
        ctx.save_for_backward(mu_e, kappa_e, res.u)
        return res.u.clone()

    @staticmethod
    def backward(ctx, gu):
        mu_e, kappa_e, u = ctx.saved_tensors
        nt = ctx.newton
        _set_params(nt.asm, None, mu_e, kappa_e)
        nt.tangent(u)
        rhs = torch.where(nt.free, gu.detach(), torch.zeros_like(gu))
        lam, _ = nt.solve_linear(rhs)
        _, gmu, gk = nt.asm.adjoint(u, lam)
        return -gmu, -gk, lam, None, None, None, None, None


def static_equilibrium(newton: DeviceNewton, mu_e, kappa_e, f_ext, n_steps: int = 1, nr_tol: float = 1e-10,
                       polish: int = 2, u0=None):
    """u*(mu_e, kappa_e, f_ext) with an adjoint backward; ``polish`` as in ``DeviceNewton.solve``.

    ``u0`` starts Newton from a nearby equilibrium (for instance that of slightly different
    moduli) instead of from zero; it is not differentiated."""
    return StaticEquilibrium.apply(mu_e, kappa_e, f_ext, newton, n_steps, nr_tol, polish, u0)


def identify_shear_moduli(newton: DeviceNewton, f_ext, obs_dofs, u_target, mu0, kappa_ratio: float = 50.0,
                          max_iter: int = 30, n_steps: int = 1, nr_tol: float = 1e-10):
    """Fit per-element shear moduli (log-parametrised) to observed displacements.

    Loss = 1/2 || u*(mu)[obs] - u_target ||^2 with kappa = kappa_ratio * mu.  Returns
    (mu, loss history).  Each loss evaluation is one forward solve and one adjoint solve.
    """
    from scipy.optimize import minimize

    dev = newton.asm.device
    obs = torch.as_tensor(np.asarray(obs_dofs), device=dev)
    tgt = torch.as_tensor(np.asarray(u_target, dtype=np.float64), device=dev)
    hist = []

    def fun(theta):
        t = torch.tensor(theta, dtype=torch.float64, device=dev, requires_grad=True)
        mu = torch.exp(t)
        u = static_equilibrium(newton, mu, kappa_ratio * mu, f_ext, n_steps=n_steps, nr_tol=nr_tol)
        loss = 0.5 * torch.sum((u[obs] - tgt) ** 2)
        loss.backward()
        hist.append(float(loss))
        return float(loss), t.grad.detach().cpu().numpy()

    r = minimize(fun, np.log(np.asarray(mu0, dtype=np.float64)), jac=True, method="L-BFGS-B",
                 options={"maxiter": max_iter})
    return np.exp(r.x), hist
