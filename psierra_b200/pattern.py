"""Mesh sparsity pattern and node graph, built once per mesh through the C ABI.

``MeshPattern`` holds the host arrays (numpy) produced by ``psx_graph_count``,
``psx_graph_fill`` and ``psx_csr_pattern`` and lazily mirrors them on the GPU.
Its ``indptr``/``indices`` are the canonical CSR index arrays scipy produces from
the reference's COO triplets (psierra ``utility/assembly.py:6-34, 75-76``), so a
values array in this order is the reference's ``K_tan.data``.
"""
from __future__ import annotations

import numpy as np

from psierra_b200._lib import check, lib, ptr


class MeshPattern:
    def __init__(self, elements: np.ndarray, n_nodes: int):
        conn = np.ascontiguousarray(elements, dtype=np.int64)
        if conn.ndim != 2 or conn.shape[1] not in (4, 10):
            raise ValueError(f"elements must be (E, 4) or (E, 10), got {conn.shape}")
        E, npe = conn.shape
        N = int(n_nodes)
        L = lib()
        nbr_ptr = np.zeros(N + 1, dtype=np.int32)
        inc_ptr = np.zeros(N + 1, dtype=np.int32)
        check(L.psx_graph_count(ptr(conn), E, npe, N, ptr(nbr_ptr), ptr(inc_ptr)), "psx_graph_count")
        nbr = np.zeros(int(nbr_ptr[-1]), dtype=np.int32)
        inc_elem = np.zeros(E * npe, dtype=np.int32)
        inc_code = np.zeros(E * npe, dtype=np.uint32)
        check(L.psx_graph_fill(ptr(conn), E, npe, N, ptr(nbr_ptr), ptr(inc_ptr), ptr(nbr), ptr(inc_elem),
                               ptr(inc_code)), "psx_graph_fill")
        nnz = 9 * int(nbr_ptr[-1])
        indptr = np.zeros(3 * N + 1, dtype=np.int32)
        indices = np.zeros(nnz, dtype=np.int32)
        check(L.psx_csr_pattern(N, ptr(nbr_ptr), ptr(nbr), ptr(indptr), ptr(indices)), "psx_csr_pattern")
        self.n_elements, self.npe, self.n_nodes = E, npe, N
        self.conn = conn
        self.nbr_ptr, self.inc_ptr, self.nbr = nbr_ptr, inc_ptr, nbr
        self.inc_elem, self.inc_code = inc_elem, inc_code
        self.indptr, self.indices = indptr, indices
        self.nnz = nnz
        deg = np.diff(nbr_ptr)
        self.max_degree = int(deg.max()) if N else 0
        self._dev: dict | None = None
        self._blocks: tuple | None = None

    @property
    def n_dofs(self) -> int:
        return 3 * self.n_nodes

    def block_lists(self) -> tuple[np.ndarray, np.ndarray]:
        """(blk_ptr, blk_src) gather lists of ``psx_block_lists`` (host, cached)."""
        if self._blocks is None:
            n_ent = int(self.nbr_ptr[-1])
            blk_ptr = np.zeros(n_ent + 1, dtype=np.int32)
            blk_src = np.zeros(self.n_elements * self.npe * self.npe, dtype=np.int32)
            check(lib().psx_block_lists(ptr(self.conn), self.n_elements, self.npe, self.n_nodes,
                                        ptr(self.nbr_ptr), ptr(self.nbr), ptr(blk_ptr), ptr(blk_src)),
                  "psx_block_lists")
            self._blocks = (blk_ptr, blk_src)
        return self._blocks

    def device(self, device) -> dict:
        """Device copies of the arrays the kernels read (uploaded once)."""
        import torch

        if self._dev is None or self._dev["device"] != torch.device(device):
            t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)  # noqa: E731
            d = {
                "device": torch.device(device),
                "conn": t(self.conn.astype(np.int32)),
                "nbr_ptr": t(self.nbr_ptr),
                "inc_ptr": t(self.inc_ptr),
                "inc_elem": t(self.inc_elem),
                "inc_code": t(self.inc_code.view(np.int32)),
                "indptr": t(self.indptr),
                "indices": t(self.indices),
            }
            self._dev = d
        return self._dev
