"""Mesh sparsity pattern and node graph, built once per mesh through the C ABI.

``MeshPattern`` holds the host arrays (numpy) produced by ``psx_graph_count``,
``psx_graph_fill`` and ``psx_csr_pattern`` and lazily mirrors them on the GPU.
Its ``indptr``/``indices`` are the canonical CSR index arrays scipy produces from
the reference's COO triplets (psierra ``utility/assembly.py:6-34, 75-76``), so a
values array in this order is the reference's ``K_tan.data``.
"""
from __future__ import annotations

import ctypes

import numpy as np

from psierra_b200 import _lib
from psierra_b200._lib import check, lib, ptr


def torch_from(a: np.ndarray, device):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).to(device)


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
        self._plan_host: dict | None = None
        self.granule, self.tile, self.tile_items, self.lag, self.lag_f, self.ring_slack = self.QUEUE[npe]
        self.blocks_per_sm = 0
        self.wait_spins = 0  # polls of one bounded wait in the persistent kernels (0 = about a second)
        # Tet4 FP32 tangent sweeps run the warp-specialised kernel (element tiles and
        # gathers in separate warps) when the plan carries the gather task list
        self.split = npe == 4

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

    # queue geometry per element type: granule (elements), element tile, item tile, lag of
    # the K queue, lag of the f / K.v queue (granules), ring slack (granules; 0 = 6).  The
    # Tet4 values are the fastest of a lag x slack sweep on the 3.07M-element cube
    # (FP32-mixed f+K and f / K.v timed separately).
    QUEUE = {4: (4096, 32, 32, 20, 16, 12), 10: (512, 8, 32, 16, 16, 0)}

    def plan_host(self) -> dict:
        """Host arrays of the gather plan (``psx_plan_fill``), built once."""
        if self._plan_host is None:
            L = lib()
            E, npe, N = self.n_elements, self.npe, self.n_nodes
            n_pairs = np.zeros(1, dtype=np.int64)
            n_src = np.zeros(1, dtype=np.int64)
            check(L.psx_plan_count(ptr(self.conn), E, npe, N, ptr(self.nbr_ptr), ptr(n_pairs), ptr(n_src)),
                  "psx_plan_count")
            P, S = int(n_pairs[0]), int(n_src[0])
            ng = (E + self.granule - 1) // self.granule
            h = {
                "pair_info": np.zeros(4 * max(P, 1), dtype=np.int32),
                "pair_ptr": np.zeros(P + 1, dtype=np.int32),
                "pair_src": np.zeros(max(S, 1), dtype=np.int32),
                "pair_gptr": np.zeros(ng + 1, dtype=np.int32),
                "node_info": np.zeros(4 * N, dtype=np.int32),
                "node_ptr": np.zeros(N + 1, dtype=np.int32),
                "node_src": np.zeros(E * npe, dtype=np.int32),
                "node_gptr": np.zeros(ng + 1, dtype=np.int32),
                "max_span": np.zeros(1, dtype=np.int64),
            }
            check(L.psx_plan_fill(ptr(self.conn), E, npe, N, ptr(self.nbr_ptr), ptr(self.nbr), self.granule,
                                  ptr(h["pair_info"]), ptr(h["pair_ptr"]), ptr(h["pair_src"]), ptr(h["pair_gptr"]),
                                  ptr(h["node_info"]), ptr(h["node_ptr"]), ptr(h["node_src"]), ptr(h["node_gptr"]),
                                  ptr(h["max_span"])), "psx_plan_fill")
            h["n_pairs"], h["n_granules"] = P, ng
            if npe == 4:
                h.update(self._tile_plan(h, P))
            self._plan_host = h
        return self._plan_host

    def _tile_plan(self, h: dict, n_pairs: int) -> dict:
        """Tile records of the Tet4 kernels (``psx_tile_plan_fill``)."""
        E, N, T = self.n_elements, self.n_nodes, self.tile
        nt = (E + T - 1) // T
        L = lib()
        stride = int(L.psx_tile_meta_stride(T))
        i32 = lambda n: np.zeros(max(int(n), 1), dtype=np.int32)  # noqa: E731
        t = {
            "tile_meta": np.zeros(nt * stride, dtype=np.uint8),
            "pair_ptr_t": i32(n_pairs + 1), "pair_src_t": i32(h["pair_src"].size),
            "node_ptr_t": i32(N + 1), "node_src_t": i32(h["node_src"].size),
        }
        caps = np.zeros(2, dtype=np.int32)
        check(L.psx_tile_plan_fill(ptr(self.conn), E, 4, T, ptr(h["pair_ptr"]), ptr(h["pair_src"]), n_pairs,
                                   ptr(h["node_ptr"]), ptr(h["node_src"]), N, ptr(t["tile_meta"]), ptr(t["pair_ptr_t"]),
                                   ptr(t["pair_src_t"]), ptr(t["node_ptr_t"]), ptr(t["node_src_t"]), ptr(caps)),
              "psx_tile_plan_fill")
        # trim the upper-bound lists to what was written
        t["pair_src_t"] = t["pair_src_t"][: max(int(t["pair_ptr_t"][-1]), 1)].copy()
        t["node_src_t"] = t["node_src_t"][: max(int(t["node_ptr_t"][-1]), 1)].copy()
        t["tile_caps"] = caps
        t["tile_meta_stride"] = stride
        return t

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
            h = self.plan_host()
            for k in ("pair_info", "pair_ptr", "pair_src", "node_info", "node_ptr", "node_src"):
                d[k] = t(h[k])
            st = _lib.PlanStruct()
            st.npe, st.n_granules = self.npe, h["n_granules"]
            st.n_elements, st.n_nodes, st.n_pairs = self.n_elements, self.n_nodes, h["n_pairs"]
            st.granule, st.max_span = self.granule, int(h["max_span"][0])
            for k in ("conn", "pair_info", "pair_ptr", "pair_src", "node_info", "node_ptr", "node_src"):
                setattr(st, k, d[k].data_ptr())
            st.pair_gptr = h["pair_gptr"].ctypes.data
            st.node_gptr = h["node_gptr"].ctypes.data
            if self.npe == 4:
                for k in ("tile_meta", "pair_ptr_t", "pair_src_t", "node_ptr_t", "node_src_t"):
                    d[k] = t(h[k])
                    setattr(st, k, d[k].data_ptr())
                st.tile_cap_pairs, st.tile_cap_nodes = int(h["tile_caps"][0]), int(h["tile_caps"][1])
            d["plan"] = st
            self._build_tasks(d)
            self._dev = d
        return self._dev

    def _build_tasks(self, d: dict) -> None:
        """(Re)build the element/gather task queues of the plan in ``d`` for the current lag."""
        t = lambda a: torch_from(a, d["device"])  # noqa: E731
        st = d["plan"]
        h = self.plan_host()
        st.tile, st.lag, st.lag_f, st.tile_items = self.tile, self.lag, self.lag_f, self.tile_items
        st.blocks_per_sm = self.blocks_per_sm
        st.ring_slack = self.ring_slack
        st.wait_spins = self.wait_spins
        L = lib()
        for key, with_pairs, lag in (("k", 1, self.lag), ("f", 0, self.lag_f)):
            nt = ctypes.c_int64()
            check(L.psx_task_count(ctypes.byref(st), with_pairs, self.tile, self.tile_items, lag,
                                   ctypes.byref(nt)), "psx_task_count")
            tasks = np.zeros(4 * max(int(nt.value), 1), dtype=np.int32)
            btiles = np.zeros(max(h["n_granules"], 1), dtype=np.int32)
            check(L.psx_task_fill(ctypes.byref(st), with_pairs, self.tile, self.tile_items, lag, ptr(tasks),
                                  ptr(btiles)), "psx_task_fill")
            d["tasks_" + key], d["btiles_" + key] = t(tasks), t(btiles)
            setattr(st, "n_tasks_" + key, int(nt.value))
            setattr(st, "tasks_" + key, d["tasks_" + key].data_ptr())
            setattr(st, "btiles_" + key, d["btiles_" + key].data_ptr())
            if key == "k" and self.npe == 4:
                # the gather tasks of the K queue in queue order (kinds 1 and 2)
                tk = tasks[: 4 * int(nt.value)].reshape(-1, 4)
                gk = np.ascontiguousarray(tk[tk[:, 0] != 0])
                d["gtasks_k"] = t(gk.reshape(-1) if gk.size else np.zeros(4, dtype=np.int32))
                d["n_gtasks_k"] = int(gk.shape[0])
        self._apply_split(d)

    def _apply_split(self, d: dict) -> None:
        st = d["plan"]
        on = self.split and d.get("n_gtasks_k", 0) > 0
        st.n_gtasks_k = d["n_gtasks_k"] if on else 0
        st.gtasks_k = d["gtasks_k"].data_ptr() if on else None

    def set_wait_limit(self, spins: int) -> None:
        """Polls after which a bounded wait of the persistent kernels gives up (0 = the
        default of 1 << 22, about a second).  A wait that gives up sets status flag bit 0,
        and the assembler then raises; the kernel itself always runs to its end."""
        if int(spins) < 0:
            raise ValueError("spins must be >= 0")
        self.wait_spins = int(spins)
        if self._dev is not None:
            self._dev["plan"].wait_spins = self.wait_spins

    def set_queue(self, lag: int | None = None, blocks_per_sm: int | None = None,
                  ring_slack: int | None = None, lag_f: int | None = None, split: bool | None = None) -> None:
        """Change the persistent launch's lags (granules; ``lag`` for the K queue, ``lag_f``
        for the f / K.v queue), blocks per SM (0 = default), ring slack (granules beyond
        span + lag; 0 = the minimum, 6) and whether Tet4 FP32 tangent sweeps run the
        warp-specialised kernel (``split``; the mixed kernel otherwise).

        Rebuilds the task queues when a lag changes; a workspace sized for the old values
        must be re-queried (``psx_work_bytes``) afterwards.
        """
        rebuild = (lag is not None and int(lag) != self.lag) or (lag_f is not None and int(lag_f) != self.lag_f)
        for v in (lag, lag_f):
            if v is not None and int(v) < 0:
                raise ValueError("lag must be >= 0")
        if lag is not None:
            self.lag = int(lag)
        if lag_f is not None:
            self.lag_f = int(lag_f)
        if blocks_per_sm is not None:
            self.blocks_per_sm = int(blocks_per_sm)
        if ring_slack is not None:
            self.ring_slack = int(ring_slack)
        if split is not None:
            self.split = bool(split) and self.npe == 4
        if self._dev is not None:
            if rebuild:
                self._build_tasks(self._dev)
            self._apply_split(self._dev)
            self._dev["plan"].blocks_per_sm = self.blocks_per_sm
            self._dev["plan"].ring_slack = self.ring_slack
