"""Tet4 F-bar (nodal volume averaging) assembly on the GPU.

Restates pSierra's ``Tet4Fbar`` (psierra ``element/tet4_fbar.py``): element forces and the
deviatoric tangent at ``F_bar = (J_bar / J)^(1/3) F`` with ``J_bar`` the element mean of
nodal volume ratios, plus the nodal volumetric blocks ``kappa v0_a g_a g_a^T`` that couple
every two nodes of a node's element patch.  The tangent therefore lives on the two-ring
node graph; ``FbarAssembler`` builds that pattern and the gather lists once per mesh
(host, C ABI) and runs the six kernels of ``psx_fbar_assemble`` per call.
"""
from __future__ import annotations

import ctypes

import numpy as np
import scipy.sparse as spsp
import torch

from psierra_b200._lib import check, lib, ptr
from psierra_b200.material import material_moduli
from psierra_b200.pattern import MeshPattern


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


class FbarAssembler:
    def __init__(self, nodes: np.ndarray, elements: np.ndarray, material, device=None):
        if not torch.cuda.is_available():
            raise RuntimeError("psierra_b200 requires a CUDA device (no CPU fallback)")
        el = np.ascontiguousarray(elements, dtype=np.int64)
        if el.ndim != 2 or el.shape[1] != 4:
            raise ValueError(f"Tet4Fbar needs (E, 4) elements, got {el.shape}")
        if getattr(material, "mu_e", None) is not None:
            raise NotImplementedError("Tet4Fbar uses one bulk modulus for its nodal blocks: scalar moduli only")
        self.device = torch.device(device if device is not None else "cuda")
        L = lib()
        nodes = np.ascontiguousarray(nodes, dtype=np.float64)
        self.n_nodes, self.n_elements = nodes.shape[0], el.shape[0]
        self.mu, self.kappa, self.lam = material_moduli(material)
        p = MeshPattern(el, self.n_nodes)
        self.pattern = p
        h = p.plan_host()
        blk_ptr, blk_src = p.block_lists()
        N = self.n_nodes
        n2, nv = ctypes.c_int64(), ctypes.c_int64()
        check(L.psx_fbar_plan_count(N, ptr(p.nbr_ptr), ptr(p.nbr), ctypes.byref(n2), ctypes.byref(nv)),
              "psx_fbar_plan_count")
        nbr2_ptr = np.zeros(N + 1, dtype=np.int32)
        nbr2 = np.zeros(max(int(n2.value), 1), dtype=np.int32)
        pair_info2 = np.zeros(max(4 * h["n_pairs"], 1), dtype=np.int32)
        node_info2 = np.zeros(4 * N, dtype=np.int32)
        vol_ptr = np.zeros(int(n2.value) + 1, dtype=np.int32)
        vol_src = np.zeros(max(3 * int(nv.value), 1), dtype=np.int32)
        check(L.psx_fbar_plan_fill(N, ptr(p.nbr_ptr), ptr(p.nbr), h["n_pairs"], ptr(h["pair_info"]),
                                   ptr(h["node_info"]), ptr(nbr2_ptr), ptr(nbr2), ptr(pair_info2), ptr(node_info2),
                                   ptr(vol_ptr), ptr(vol_src)), "psx_fbar_plan_fill")
        self.nnz = 9 * int(n2.value)
        self.indptr = np.zeros(3 * N + 1, dtype=np.int32)
        self.indices = np.zeros(self.nnz, dtype=np.int32)
        check(L.psx_csr_pattern(N, ptr(nbr2_ptr), ptr(nbr2), ptr(self.indptr), ptr(self.indices)), "psx_csr_pattern")
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(self.device)  # noqa: E731
        self.d = {
            "conn": t(el.astype(np.int32)), "X": t(nodes), "inc_ptr": t(p.inc_ptr), "inc_elem": t(p.inc_elem),
            "nbr_ptr": t(p.nbr_ptr), "nbr": t(p.nbr), "blk_ptr": t(blk_ptr), "blk_src": t(blk_src),
            "pair_info2": t(pair_info2), "pair_ptr": t(h["pair_ptr"]), "pair_src": t(h["pair_src"]),
            "node_info2": t(node_info2), "node_ptr": t(h["node_ptr"]), "node_src": t(h["node_src"]),
            "nbr2_ptr": t(nbr2_ptr), "vol_ptr": t(vol_ptr), "vol_src": t(vol_src),
        }
        self.device = self.d["X"].device  # resolved index ("cuda" -> "cuda:0")
        self.n_pairs = h["n_pairs"]
        self.n_nbr = int(p.nbr_ptr[-1])
        nw = int(L.psx_fbar_work_doubles(self.n_elements, N, self.n_nbr))
        self.work = torch.empty(nw, dtype=torch.float64, device=self.device)
        nbytes = int(L.psx_status_bytes())
        self.status = torch.zeros((nbytes + 3) // 4, dtype=torch.int32, device=self.device)
        self.jbar = torch.empty(self.n_elements, dtype=torch.float64, device=self.device)

    @property
    def n_dofs(self) -> int:
        return 3 * self.n_nodes

    def assemble(self, u: torch.Tensor, want_f: bool = True, want_k: bool = True, jbar: torch.Tensor | None = None,
                 check_status: bool = True):
        """``(f (3N), k (nnz two-ring values))`` on the device; either may be None."""
        if not (want_f or want_k):
            raise ValueError("nothing requested")
        u = u.reshape(-1).contiguous()
        if u.dtype != torch.float64 or u.numel() != 3 * self.n_nodes or u.device != self.device:
            raise ValueError("u must be a float64 (3N,) tensor on the assembler's device")
        f = torch.empty(3 * self.n_nodes, dtype=torch.float64, device=self.device) if want_f else None
        k = torch.empty(self.nnz, dtype=torch.float64, device=self.device) if want_k else None
        self.status.zero_()
        d = self.d
        check(lib().psx_fbar_assemble(
            ptr(d["conn"]), self.n_elements, self.n_nodes, ptr(d["X"]), ptr(u), self.mu, self.kappa, ptr(d["inc_ptr"]),
            ptr(d["inc_elem"]), ptr(d["nbr_ptr"]), ptr(d["nbr"]), self.n_nbr, ptr(d["blk_ptr"]), ptr(d["blk_src"]),
            self.n_pairs, ptr(d["pair_info2"]), ptr(d["pair_ptr"]), ptr(d["pair_src"]), ptr(d["node_info2"]),
            ptr(d["node_ptr"]), ptr(d["node_src"]), ptr(d["nbr2_ptr"]), ptr(d["vol_ptr"]), ptr(d["vol_src"]),
            ptr(jbar), ptr(f), ptr(k), self.nnz, ptr(self.jbar), ptr(self.work), self.work.numel(), ptr(self.status),
            _stream()), "psx_fbar_assemble")
        if check_status:
            self.raise_on_bad_elements(u)
        return f, k

    def raise_on_bad_elements(self, u: torch.Tensor) -> None:
        s = self.status[:4].cpu().numpy()
        if s[0] == 0 and s[1] == 0:
            return
        e = int(0x7FFFFFFF - int(s[2]))
        el = self.d["conn"][e].long().cpu().numpy()
        X = self.d["X"].cpu().numpy()[el]
        A = np.ones((4, 4))
        A[:, 1:] = X
        detA = float(np.linalg.det(A))
        if s[1]:
            raise ValueError(f"Negative or zero element volume detected (det(A) = {detA}). "
                             "Check element vertex ordering.")
        Un = u.reshape(-1, 3).cpu().numpy()[el]
        H = np.linalg.inv(A)[1:, :].T
        J = float(np.linalg.det(np.eye(3) + Un.T @ H))
        raise ValueError(f"Element inversion detected at element {e}: det(F) = {J:.4e} <= 0.")

    def csr(self, k: torch.Tensor) -> spsp.csr_matrix:
        """Host CSR with the reference's pattern: scipy's ``K_dev + K_vol`` drops exact zeros."""
        A = spsp.csr_matrix((k.cpu().numpy(), self.indices, self.indptr), shape=(self.n_dofs,) * 2)
        A.eliminate_zeros()
        return A

    def element_matrices(self, X_elem: np.ndarray, u_elem: np.ndarray, jbar: np.ndarray):
        """Independent elements with given J_bar: ``(k (n,12,12), f (n,12))`` (host arrays)."""
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(self.device)  # noqa: E731
        Xd, ud, jd = t(X_elem), t(u_elem), t(np.atleast_1d(jbar))
        n = jd.numel()
        k = torch.empty((n, 12, 12), dtype=torch.float64, device=self.device)
        f = torch.empty((n, 12), dtype=torch.float64, device=self.device)
        self.status.zero_()
        check(lib().psx_fbar_element(n, ptr(Xd), ptr(ud), ptr(jd), self.mu, self.kappa, ptr(k), ptr(f),
                                     ptr(self.status), _stream()), "psx_fbar_element")
        s = self.status[:4].cpu().numpy()
        if s[0] or s[1]:
            e = int(0x7FFFFFFF - int(s[2]))
            X = np.asarray(X_elem, dtype=np.float64).reshape(-1, 4, 3)[e]
            A = np.ones((4, 4))
            A[:, 1:] = X
            if s[1]:
                raise ValueError(f"Negative or zero element volume detected (det(A) = {np.linalg.det(A)}). "
                                 "Check element vertex ordering.")
            H = np.linalg.inv(A)[1:, :].T
            Un = np.asarray(u_elem, dtype=np.float64).reshape(-1, 4, 3)[e]
            J = float(np.linalg.det(np.eye(3) + Un.T @ H))
            raise ValueError(f"Element inversion detected: det(F) = {J:.4e} <= 0.")
        return k.cpu().numpy(), f.cpu().numpy()
