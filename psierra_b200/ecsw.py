"""Hyper-reduced (ECSW) evaluation of the Tet4 NeoHookean model on the GPU.

Mirrors ``HyperReducedECSWModel.evaluate_forces_and_stiffness`` (psierra
``hyperreduction/model.py:254-318``): only the elements of the reduced integration domain
(RID) are evaluated, each at ``u_e = Phi_e u_r`` with its cubature weight, and projected
onto the modal basis.  ``ECSWEvaluator`` caches the RID's reference coordinates, modal
sub-bases and weights on the device once (``model.py:181-206``); one evaluation is two
kernel launches (``psx_ecsw_evaluate``).
"""
from __future__ import annotations

import numpy as np
import torch

from psierra_b200._lib import check, lib, ptr
from psierra_b200.material import _host, material_moduli


class ECSWEvaluator:
    def __init__(self, nodes, elements, material, basis_matrix, element_indices, weights, device=None):
        if not torch.cuda.is_available():
            raise RuntimeError("psierra_b200 requires a CUDA device (no CPU fallback)")
        el = np.asarray(elements, dtype=np.int64)
        if el.ndim != 2 or el.shape[1] != 4:
            raise ValueError("the ECSW evaluator covers Tet4 meshes")
        idx = np.asarray(element_indices, dtype=np.int64).ravel()
        w = np.asarray(weights, dtype=np.float64).ravel()
        if idx.size != w.size or idx.size == 0:
            raise ValueError("element_indices and weights must be non-empty and of equal length")
        Phi = np.asarray(basis_matrix, dtype=np.float64)
        self.r = Phi.shape[1]
        dev = torch.device(device if device is not None else "cuda")
        nodes = np.asarray(nodes, dtype=np.float64)
        rid_nodes = el[idx]                                                  # (p, 4)
        edofs = (3 * rid_nodes[:, :, None] + np.arange(3)).reshape(-1, 12)   # (p, 12)
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(dev)  # noqa: E731
        self.X = t(nodes[rid_nodes].reshape(-1, 12))
        self.phi = t(Phi[edofs])                                             # (p, 12, r)
        self.w = t(w)
        self.mu, self.kappa, _ = material_moduli(material)
        mu_e = getattr(material, "mu_e", None)
        self.mu_e = t(np.asarray(_host(mu_e))[idx]) if mu_e is not None else None
        self.kappa_e = t(np.asarray(_host(material.kappa_e))[idx]) if mu_e is not None else None
        self.n = idx.size
        self.device = self.X.device
        self.work = torch.empty(int(lib().psx_ecsw_work_doubles(self.n, self.r)), dtype=torch.float64, device=dev)
        self.status = torch.zeros((int(lib().psx_status_bytes()) + 3) // 4, dtype=torch.int32, device=dev)

    def evaluate_device(self, u_r: torch.Tensor):
        """``(f_r (r,), K_r (r, r))`` as device tensors for a device ``u_r``."""
        u_r = u_r.to(self.device, torch.float64).contiguous()
        f = torch.empty(self.r, dtype=torch.float64, device=self.device)
        K = torch.empty((self.r, self.r), dtype=torch.float64, device=self.device)
        self.status.zero_()
        check(lib().psx_ecsw_evaluate(self.n, self.r, ptr(self.X), ptr(self.phi), ptr(self.w), ptr(u_r),
                                      ptr(self.mu_e), ptr(self.kappa_e), self.mu, self.kappa, ptr(f), ptr(K),
                                      ptr(self.work), self.work.numel(), ptr(self.status),
                                      torch.cuda.current_stream().cuda_stream), "psx_ecsw_evaluate")
        s = self.status[:3].cpu().numpy()
        if s[0] or s[1]:
            e = int(0x7FFFFFFF - int(s[2]))
            X = self.X[e].cpu().numpy().reshape(4, 3)
            A = np.ones((4, 4))
            A[:, 1:] = X
            if s[1]:
                raise ValueError(f"Negative or zero element volume detected (det(A) = {np.linalg.det(A)}). "
                                 "Check element vertex ordering.")
            un = (self.phi[e] @ u_r).cpu().numpy().reshape(4, 3)
            J = float(np.linalg.det(np.eye(3) + un.T @ np.linalg.inv(A)[1:, :].T))
            raise ValueError(f"Element inversion detected: det(F) = {J:.4e} <= 0.")
        return f, K

    def evaluate_forces_and_stiffness(self, u_r) -> tuple[np.ndarray, np.ndarray]:
        """Host arrays, as the reference method returns them."""
        u = np.asarray(u_r, dtype=np.float64).ravel()
        if u.size != self.r:
            raise ValueError(f"u_r size ({u.size}) must match reduced dimension ({self.r}).")
        f, K = self.evaluate_device(torch.from_numpy(u).to(self.device))
        return f.cpu().numpy(), K.cpu().numpy()
