"""Two-level preconditioner: block-Jacobi plus a coarse space of rigid-body modes.

No counterpart in the reference, whose CG (psierra ``solver/sparse_linear_solver.py:37-68``)
uses the Jacobi operator and which suggests a stronger preconditioner for large meshes.
Block-Jacobi CG needs O(10^4) iterations on slender beams: their bending modes are
global and the iteration propagates them one element per step.  This adds the coarse
correction of a two-level additive Schwarz method:

    M^-1 r = B^-1 r + P A_c^-1 P^T r,     A_c = P^T A P,

with B the node blocks of A and P six columns per aggregate of nodes (three
translations, three rotations about the aggregate's centroid: a rigid motion of the
aggregate).  Aggregates are slices of each mesh instance along its longest principal
axis, a few cross-sections each (sized by positions along the axis, not by node count, so
that a thin beam gets as many slices as a thick one), so that a beam's coarse space
carries its bending and torsion, which block-Jacobi resolves slowest.

A_c changes with every tangent.  It is assembled on the device by probing: the
aggregates are coloured so that two aggregates of one colour are never both coupled to a
third (a distance-2 colouring of the aggregate graph).  Then, for every colour c and mode s,
one product w = A (sum of the columns (a, s) of the aggregates of colour c) and one
restriction P^T w give, for every aggregate b, the entries A_c[(b, t), (a, s)] of the one
aggregate a of colour c coupled to b.  Every entry is written once, so A_c is
reproducible.  The instances of a batch are independent blocks of A_c; each block is
factorised and inverted densely (``torch.linalg.cholesky_ex``, no host
synchronisation, so the update can be captured in a CUDA graph), and the CG applies the
inverse as a matrix-vector product (``psx_pcg_coarse``).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from psierra_b200 import _lib
from psierra_b200._lib import CoarseStruct, check, lib, ptr


def slice_aggregates(nodes: np.ndarray, node_offsets, levels_per_aggregate: int = 4, max_aggregates: int = 64):
    """Aggregate of every node: per instance (nodes node_offsets[i]:node_offsets[i+1]),
    slices of roughly equal node count along the instance's longest principal axis, each
    about ``levels_per_aggregate`` distinct positions along it (cross-sections of a
    structured mesh), at most ``max_aggregates`` per instance.  Nodes with the same
    coordinate along the axis share a slice.  Returns (node_agg (N,), block_agg (B+1,)),
    aggregates numbered instance by instance."""
    X = np.asarray(nodes, dtype=np.float64)
    offs = np.asarray(node_offsets, dtype=np.int64)
    node_agg = np.empty(X.shape[0], dtype=np.int64)
    block_agg = [0]
    for b in range(len(offs) - 1):
        lo, hi = int(offs[b]), int(offs[b + 1])
        Y = X[lo:hi] - X[lo:hi].mean(axis=0)
        w, v = np.linalg.eigh(Y.T @ Y)
        t = Y @ v[:, np.argmax(w)]
        # levels: positions along the axis equal to 1e-9 of the extent (a cross-section
        # of a structured mesh is one level), never split between slices
        span = max(float(np.ptp(t)), 1e-300)
        levels, inv, counts = np.unique(np.round(t / (1e-9 * span)), return_inverse=True, return_counts=True)
        n = hi - lo
        n_agg = min(max_aggregates, max(1, int(round(len(levels) / max(1, levels_per_aggregate)))))
        mid = np.cumsum(counts) - 0.5 * counts  # node rank at the middle of each level
        level_agg = np.minimum((mid * n_agg / n).astype(np.int64), n_agg - 1)
        used, a = np.unique(level_agg[inv], return_inverse=True)  # drop empty slices
        node_agg[lo:hi] = block_agg[-1] + a
        block_agg.append(block_agg[-1] + len(used))
    return node_agg, np.asarray(block_agg, dtype=np.int64)


def aggregate_graph(elements: np.ndarray, node_agg: np.ndarray, n_agg: int):
    """Sorted neighbour lists (including itself) of every aggregate: a and b are coupled
    when an element has nodes in both."""
    ea = np.asarray(node_agg, dtype=np.int64)[np.asarray(elements, dtype=np.int64)]
    npe = ea.shape[1]
    keys = [np.arange(n_agg, dtype=np.int64) * (n_agg + 1)]
    for i in range(npe):
        for j in range(npe):
            if i != j:
                k = ea[:, i] * n_agg + ea[:, j]
                keys.append(np.unique(k[ea[:, i] != ea[:, j]]))
    keys = np.unique(np.concatenate(keys))
    rows, cols = keys // n_agg, keys % n_agg
    ptr_ = np.searchsorted(rows, np.arange(n_agg + 1))
    return ptr_, cols


def distance2_colouring(ptr_: np.ndarray, nbr: np.ndarray) -> np.ndarray:
    """Greedy colouring in index order such that aggregates sharing a neighbour (or
    coupled directly) get different colours."""
    n = len(ptr_) - 1
    colour = np.full(n, -1, dtype=np.int64)
    for a in range(n):
        taken = set()
        for b in nbr[ptr_[a]:ptr_[a + 1]]:
            for c in nbr[ptr_[b]:ptr_[b + 1]]:
                if colour[c] >= 0:
                    taken.add(int(colour[c]))
        k = 0
        while k in taken:
            k += 1
        colour[a] = k
    return colour


class CoarseSpace:
    """Rigid-body-mode coarse space of a (batch of) mesh(es) on the device.

    ``fixed``: (3N,) nonzero on eliminated DOFs (rows of P there are zero);
    ``node_offsets``: instance boundaries in the node numbering (one instance if None).
    ``update(k, indptr, indices)`` refreshes A_c^-1 from an eliminated tangent;
    ``struct`` is the ``psx_coarse_t`` the CG takes.
    """

    def __init__(self, nodes, elements, fixed, node_offsets=None, levels_per_aggregate: int = 4,
                 max_aggregates: int = 64, device=None) -> None:
        X = np.asarray(nodes, dtype=np.float64)
        N = X.shape[0]
        offs = np.asarray([0, N] if node_offsets is None else node_offsets, dtype=np.int64)
        node_agg, block_agg = slice_aggregates(X, offs, levels_per_aggregate, max_aggregates)
        n_agg = int(block_agg[-1])
        order = np.argsort(node_agg, kind="stable")
        agg_ptr = np.searchsorted(node_agg[order], np.arange(n_agg + 1))
        cent = np.zeros((n_agg, 3))
        np.add.at(cent, node_agg, X)
        cent /= np.diff(agg_ptr)[:, None]
        d = X - cent[node_agg]
        gptr, gnbr = aggregate_graph(elements, node_agg, n_agg)
        colour = distance2_colouring(gptr, gnbr)
        n_col = int(colour.max()) + 1
        block_of = np.repeat(np.arange(len(block_agg) - 1), np.diff(block_agg))
        local = np.arange(n_agg) - block_agg[block_of]
        nc = 6 * int(np.diff(block_agg).max())
        # probing targets: for colour c, aggregate b gets the columns of its coupled
        # aggregate a of colour c (unique by the colouring)
        self.targets = []
        for c in range(n_col):
            bs, as_ = [], []
            for b in range(n_agg):
                nb = gnbr[gptr[b]:gptr[b + 1]]
                hit = nb[colour[nb] == c]
                assert len(hit) <= 1
                if len(hit):
                    bs.append(b)
                    as_.append(int(hit[0]))
            self.targets.append((np.asarray(bs, dtype=np.int64), np.asarray(as_, dtype=np.int64)))
        dev = torch.device("cuda") if device is None else torch.device(device)
        i32 = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.int32)).to(dev)  # noqa: E731
        self.device = dev
        self.n_nodes, self.n_agg, self.n_blocks, self.nc, self.n_colours = N, n_agg, len(block_agg) - 1, nc, n_col
        self.node_agg = i32(node_agg)
        self.agg_ptr = i32(agg_ptr)
        self.agg_nodes = i32(order)
        self.block_agg = i32(block_agg)
        self.agg_colour = i32(colour)
        self.d = torch.from_numpy(np.ascontiguousarray(d)).to(dev)
        self.fixed = torch.as_tensor(np.asarray(fixed, dtype=np.uint8)).to(dev)
        f64 = dict(dtype=torch.float64, device=dev)
        self.ainv = torch.zeros((self.n_blocks, nc, nc), **f64)
        self.ac = torch.zeros((self.n_blocks, nc, nc), **f64)
        self.rc = torch.zeros(6 * n_agg, **f64)
        self.yc = torch.zeros(6 * n_agg, **f64)
        self.v = torch.zeros(3 * N, **f64)
        self.w = torch.zeros(3 * N, **f64)
        self.r6 = torch.zeros(6 * n_agg, **f64)
        # index tensors that scatter a restriction into A_c: entry (b, t) of the probe
        # (c, s) lands at block(b), row 6 local(b) + t, column 6 local(a) + s
        self._scatter = []
        for c, (bs, as_) in enumerate(self.targets):
            per_mode = []
            for s in range(6):
                t = np.arange(6)
                blk = np.repeat(block_of[bs], 6)
                row = (6 * local[bs][:, None] + t[None, :]).reshape(-1)
                col = np.repeat(6 * local[as_] + s, 6)
                src = (6 * bs[:, None] + t[None, :]).reshape(-1)
                per_mode.append(tuple(torch.from_numpy(x.astype(np.int64)).to(dev) for x in (blk, row, col, src)))
            self._scatter.append(per_mode)
        sizes = 6 * np.diff(block_agg)
        pad = np.zeros((self.n_blocks, nc), dtype=bool)
        for b in range(self.n_blocks):
            pad[b, sizes[b]:] = True
        self._pad = torch.from_numpy(pad).to(dev)
        self._eye = torch.eye(nc, **f64).expand(self.n_blocks, nc, nc).contiguous()
        self.struct = CoarseStruct(N, n_agg, ptr(self.node_agg), ptr(self.agg_ptr), ptr(self.agg_nodes), ptr(self.d),
                                   ptr(self.fixed), self.n_blocks, nc, ptr(self.block_agg), ptr(self.ainv),
                                   ptr(self.rc), ptr(self.yc))

    def probe(self, colour: int, mode: int, out: torch.Tensor) -> torch.Tensor:
        check(lib().psx_coarse_probe(self.struct_ptr(), ptr(self.agg_colour), colour, mode, ptr(out),
                                     torch.cuda.current_stream().cuda_stream), "psx_coarse_probe")
        return out

    def restrict(self, w: torch.Tensor, out: torch.Tensor) -> torch.Tensor:
        check(lib().psx_coarse_restrict(self.struct_ptr(), ptr(w), ptr(out), torch.cuda.current_stream().cuda_stream),
              "psx_coarse_restrict")
        return out

    def struct_ptr(self):
        """``psx_coarse_t*`` for the C ABI."""
        return ctypes.byref(self.struct)

    def update(self, k: torch.Tensor, indptr: torch.Tensor, indices: torch.Tensor) -> None:
        """A_c = P^T K P by probing, then A_c^-1 per block, all on the current stream."""
        vp = _lib.PSX_FP64 if k.dtype == torch.float64 else _lib.PSX_FP32_MIXED
        stream = torch.cuda.current_stream().cuda_stream
        n = 3 * self.n_nodes
        self.ac.zero_()
        for c in range(self.n_colours):
            for s in range(6):
                if self._scatter[c][s][0].numel() == 0:
                    continue
                self.probe(c, s, self.v)
                check(lib().psx_csr_spmv(n, ptr(indptr), ptr(indices), ptr(k), vp, ptr(self.v), 1.0, 0.0, ptr(self.w),
                                         stream), "psx_csr_spmv")
                self.restrict(self.w, self.r6)
                self.fill(c, s, self.r6)
        self.invert()

    def fill(self, colour: int, mode: int, r6: torch.Tensor) -> None:
        """Write the restriction P^T A (columns (a, mode) of the aggregates a of
        ``colour``) into A_c: each entry is written once."""
        blk, row, col, src = self._scatter[colour][mode]
        self.ac.index_put_((blk, row, col), r6[src])

    def invert(self) -> None:
        """A_c^-1 of every block from ``self.ac`` (no host synchronisation)."""
        # symmetrise (probing gives both triangles; their rounding differs slightly),
        # make padded and all-fixed coarse unknowns identity rows, and factorise
        a = 0.5 * (self.ac + self.ac.transpose(1, 2))
        diag = torch.diagonal(a, dim1=1, dim2=2)
        scale = diag.abs().amax(dim=1, keepdim=True).clamp_min(1e-300)
        dead = self._pad | (diag.abs() <= 1e-13 * scale)
        keep = (~dead).to(a.dtype)
        a = a * keep[:, :, None] * keep[:, None, :]
        a = a + torch.diag_embed(dead.to(a.dtype) + 1e-12 * scale * keep)
        L, info = torch.linalg.cholesky_ex(a)
        # A^-1 = L^-T L^-1 from one batched triangular solve (cuBLAS, capturable)
        Li = torch.linalg.solve_triangular(L, self._eye, upper=False)
        torch.bmm(Li.transpose(1, 2), Li, out=self.ainv)
        # a block whose A_c is not positive definite (a tangent that lost definiteness)
        # gets no coarse correction: that instance runs plain block-Jacobi
        # (a failed factor may hold NaN, which a multiplication by zero would keep)
        use = (keep[:, :, None] * keep[:, None, :] > 0) & (info == 0)[:, None, None]
        torch.where(use, self.ainv, torch.zeros((), dtype=a.dtype, device=a.device), out=self.ainv)
        self.factor_ok = info == 0
