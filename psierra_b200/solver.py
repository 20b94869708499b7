"""Linear solvers plugged into the Newton drivers through ``SparseLinearSolver.solve(A, b)``.

``ConjugateGradientSolver`` mirrors pSierra's class of the same name (psierra
``solver/sparse_linear_solver.py:37-68``: constructor arguments, Jacobi default, the
``RuntimeError`` on non-convergence) but runs the iteration on the GPU through
``psx_pcg``: the same recurrence as ``scipy.sparse.linalg.cg`` with x0 = 0 and the
stopping test ||r|| < max(atol, rtol ||b||), with every dot product reduced in a
fixed order.  It also offers a 3x3 block-Jacobi preconditioner for node-aligned
systems and ``solve_device`` for device-resident callers.

``DirectSolver`` is the reference's SuperLU solver (``sparse_linear_solver.py:10-19``),
kept as the host-side default the drivers fall back to when no solver is given; it is
the oracle the GPU CG is checked against, not a GPU path.
"""
from __future__ import annotations

import ctypes

import numpy as np
import scipy.sparse as spsp
import torch

from psierra_b200 import _lib
from psierra_b200._lib import check, lib, ptr

PRECONDITIONERS = {None: _lib.PSX_PRECOND_NONE, "jacobi": _lib.PSX_PRECOND_JACOBI,
                   "block-jacobi": _lib.PSX_PRECOND_BJACOBI}


class SparseLinearSolver:
    """Base class (psierra ``solver/base.py:6-10``)."""

    def solve(self, A, b):  # pragma: no cover - interface
        raise NotImplementedError("Subclasses must implement solve.")


class DirectSolver(SparseLinearSolver):
    """SuperLU via ``scipy.sparse.linalg.spsolve`` (psierra ``sparse_linear_solver.py:10-19``)."""

    def solve(self, A, b):
        import scipy.sparse.linalg as spla

        if not isinstance(A, spsp.csc_matrix):
            A = A.tocsc()
        return spla.spsolve(A, b)


class PCGResult:
    def __init__(self, iterations: int, converged: bool, residual_norm: float, flags: int):
        self.iterations, self.converged, self.residual_norm, self.flags = iterations, converged, residual_norm, flags


def is_nodal_csr(indptr, indices) -> bool:
    """Whether a CSR pattern is node-blocked: the three rows of node i have the same
    columns, in triples 3j, 3j+1, 3j+2 per neighbour j (the layout ``psx_csr_pattern``
    builds, and the one ``PSX_PCG_NODAL`` asks for)."""
    indptr = np.asarray(indptr, dtype=np.int64)
    indices = np.asarray(indices, dtype=np.int64)
    n = indptr.size - 1
    if n <= 0 or n % 3 or indptr[0] != 0 or indices.size < indptr[-1]:
        return False
    lens = np.diff(indptr)
    l3 = lens.reshape(-1, 3)
    if (lens % 3).any() or not (l3 == l3[:, :1]).all():
        return False
    t = indices[: indptr[-1]].reshape(-1, 3)
    if (t[:, 0] % 3).any() or (t[:, 1] != t[:, 0] + 1).any() or (t[:, 2] != t[:, 0] + 2).any():
        return False
    c = t[:, 0]
    d = l3[:, 0] // 3  # neighbours of each node
    if d.sum() == 0:
        return True
    start = indptr[0:-1:3] // 3  # first triple of row 3i
    pos = np.repeat(start, d) + (np.arange(d.sum()) - np.repeat(np.cumsum(d) - d, d))
    dd = np.repeat(d, d)
    return bool((c[pos + dd] == c[pos]).all() and (c[pos + 2 * dd] == c[pos]).all())


class ConjugateGradientSolver(SparseLinearSolver):
    """GPU preconditioned CG with the reference solver's interface and error behaviour."""

    def __init__(self, tolerance: float = 1e-8, max_iterations: int = 2000, preconditioner="jacobi",
                 device=None, atol: float = 0.0) -> None:
        if preconditioner not in PRECONDITIONERS:
            raise ValueError(f"preconditioner must be one of {list(PRECONDITIONERS)}, got {preconditioner!r}")
        self.tolerance = tolerance
        self.max_iterations = max_iterations
        self.preconditioner = preconditioner
        self.atol = atol
        self.device = torch.device(device if device is not None else "cuda")
        self.last: PCGResult | None = None
        self._status = None
        self._work: torch.Tensor | None = None

    def _workspace(self, n: int, precond: int) -> torch.Tensor:
        nbytes = ctypes.c_int64()
        check(lib().psx_pcg_work_bytes(n, precond, ctypes.byref(nbytes)), "psx_pcg_work_bytes")
        if self._work is None or self._work.numel() < nbytes.value:
            self._work = torch.empty(int(nbytes.value), dtype=torch.uint8, device=self.device)
        return self._work

    def solve_device(self, indptr: torch.Tensor, indices: torch.Tensor, values: torch.Tensor, b: torch.Tensor,
                     x: torch.Tensor, nodal: bool = False, coarse=None) -> PCGResult:
        """Solve in place on device tensors (``x`` holds the initial guess on entry).

        ``nodal``: the CSR is node-blocked (``is_nodal_csr``; every matrix of the
        assembler's pattern is), so the SpMVs read each neighbour's columns once per node.
        ``coarse``: a ``psierra_b200.coarse.CoarseSpace`` already updated from ``values``;
        its rigid-body-mode correction is added to the block-Jacobi preconditioner.
        """
        n = b.numel()
        precond = PRECONDITIONERS[self.preconditioner]
        if precond == _lib.PSX_PRECOND_BJACOBI and n % 3:
            raise ValueError("block-jacobi needs a node-aligned system (n % 3 == 0)")
        if nodal:
            if n % 3:
                raise ValueError("a node-blocked system has n % 3 == 0")
            precond |= _lib.PSX_PCG_NODAL
        vp = _lib.PSX_FP64 if values.dtype == torch.float64 else _lib.PSX_FP32_MIXED
        if values.dtype not in (torch.float64, torch.float32):
            raise ValueError("values must be float64 or float32")
        if self._status is None:
            self._status = torch.zeros(8, dtype=torch.int32, device=self.device)
        work = self._workspace(n, precond)
        if coarse is not None:
            if (precond & ~_lib.PSX_PCG_NODAL) != _lib.PSX_PRECOND_BJACOBI:
                raise ValueError("the coarse correction is added to the block-jacobi preconditioner")
            check(lib().psx_pcg_coarse(n, ptr(indptr), ptr(indices), ptr(values), vp, ptr(b), ptr(x),
                                       float(self.tolerance), float(self.atol), int(self.max_iterations), precond,
                                       coarse.struct_ptr(), ptr(work), work.numel(), ptr(self._status),
                                       torch.cuda.current_stream().cuda_stream, 1), "psx_pcg_coarse")
        else:
            check(lib().psx_pcg(n, ptr(indptr), ptr(indices), ptr(values), vp, ptr(b), ptr(x), float(self.tolerance),
                                float(self.atol), int(self.max_iterations), precond, ptr(work), work.numel(),
                                ptr(self._status), torch.cuda.current_stream().cuda_stream), "psx_pcg")
        st = self._status.cpu()
        iters, flags = int(st[4]), int(st[5])
        rn = float(st.view(torch.float64)[3])
        self.last = PCGResult(iters, flags == 0, rn, flags)
        return self.last

    def solve(self, A, b) -> np.ndarray:
        """``A x = b`` for a scipy sparse ``A`` (host arrays in and out), x0 = 0."""
        if not isinstance(A, spsp.csr_matrix):
            A = A.tocsr()
        if not A.has_sorted_indices:
            A = A.sorted_indices()
        dev = self.device
        indptr = torch.from_numpy(np.ascontiguousarray(A.indptr, dtype=np.int32)).to(dev)
        indices = torch.from_numpy(np.ascontiguousarray(A.indices, dtype=np.int32)).to(dev)
        values = torch.from_numpy(np.ascontiguousarray(A.data, dtype=np.float64)).to(dev)
        bd = torch.from_numpy(np.ascontiguousarray(b, dtype=np.float64)).to(dev)
        x = torch.zeros_like(bd)
        res = self.solve_device(indptr, indices, values, bd, x, nodal=is_nodal_csr(A.indptr, A.indices))
        if not res.converged:
            info = self.max_iterations if res.flags == 2 else -1
            raise RuntimeError(f"Conjugate Gradient did not converge (info={info}).")
        return x.cpu().numpy()
