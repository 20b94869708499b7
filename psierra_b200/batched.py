"""Many uneven meshes in one launch, and their Newton solves as one CUDA graph.

pSierra solves one mesh per ``NonlinearStaticAnalysis`` (psierra
``analysis/nonlinear_static.py:250-404``); a study over many specimens loops over
them in Python.  Here a batch of Tet4 meshes becomes the disjoint union of their
meshes (``meshgen.concat_meshes``) with per-element moduli, so one persistent
``psx_tet4_assemble`` launch evaluates every element of every instance, whatever the
instance sizes, and the union's CSR pattern is block diagonal by construction.

``BatchedNewton`` runs the incremental Newton of every instance at once.  One Newton
iteration for the whole batch is one replay of a captured CUDA graph:

  fused f_int + K_T assembly -> symmetric elimination of the clamped DOFs ->
  R = lambda f_ext - f_int on the free DOFs -> per-instance ||R|| (fixed-order segment
  sums) -> instance mask (||R_i|| >= tol_i) -> rhs R_i / ref_i on active instances ->
  PCG with a fixed trip count (block-Jacobi, or block-Jacobi with the rigid-body-mode
  coarse correction of ``psierra_b200.coarse``, whose coarse matrices are refreshed from
  the new tangent inside the same replay) -> du_i = ref_i * solution -> u += du.

The system is block diagonal.  By default it is solved as one independent CG per
instance in the same launches (``psx_pcg_batched``: per-instance step lengths, residual
test and iteration count), so each instance converges at its own rate; one CG over the
whole system (``per_instance_cg=False``) shares its step lengths and converges at the rate
of the worst-conditioned instance.  Instance i's right-hand side is scaled by 1/ref_i
(ref_i = ||lambda f_ext,i||), which gives every instance the same relative accuracy in
the shared CG as well.  An instance that has converged (or failed) gets a zero
right-hand side, and CG then leaves its block of the solution exactly zero, so it stays
frozen as the reference's loop would leave it.  The host reads the B residual norms
once per replay to decide convergence; nothing else leaves the device.  Each replay is
also a trial: an instance whose residual turned non-finite (an inverted element) or grew
more than a hundredfold goes back to half of its step, as the reference's line search
contracts on inversion (``analysis/line_search.py:120-260``).  A non-converged instance keeps its last
converged load step, as ``NonlinearStaticAnalysis`` returns it.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np
import torch

from psierra_b200 import _lib
from psierra_b200._lib import check, lib, ptr
from psierra_b200.assembler import GPUAssembler, raise_if_wait_gave_up
from psierra_b200.material import NeoHookeanField
from psierra_b200.meshgen import concat_meshes


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def partition_instances(sizes, world: int) -> list[np.ndarray]:
    """Split a batch across ``world`` ranks (one GPU each), balanced by element count.

    Instances are independent, so each rank solves its own share with no collective on
    the data path.  Greedy longest-processing-time assignment in a fixed order (sizes
    descending, ties by index), so every rank computes the same partition; each rank's
    indices are returned ascending.
    """
    sizes = np.asarray(sizes, dtype=np.int64)
    if world <= 0:
        raise ValueError("world must be positive")
    order = np.lexsort((np.arange(sizes.size), -sizes))
    load = np.zeros(world, dtype=np.int64)
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = int(np.argmin(load))  # lowest rank wins ties
        parts[r].append(int(i))
        load[r] += sizes[i]
    return [np.array(sorted(p), dtype=np.int64) for p in parts]


class MeshBatch:
    """Disjoint union of Tet4 meshes with per-instance (or per-element) NeoHookean moduli."""

    def __init__(self, meshes, mu, kappa, precision: str = "fp32-mixed", device=None):
        if len(meshes) == 0:
            raise ValueError("empty batch")
        union, node_off, elem_off = concat_meshes(meshes)
        self.B = len(meshes)
        self.node_offsets, self.element_offsets = node_off, elem_off
        self.dof_offsets = 3 * node_off
        ne = np.diff(elem_off)
        mu_e = np.concatenate([np.broadcast_to(np.asarray(m, dtype=np.float64), (int(ne[i]),))
                               for i, m in enumerate(mu)])
        ka_e = np.concatenate([np.broadcast_to(np.asarray(k, dtype=np.float64), (int(ne[i]),))
                               for i, k in enumerate(kappa)])
        self.mesh = union
        self.asm = GPUAssembler(union.nodes, union.elements, NeoHookeanField(mu_e, ka_e), precision=precision,
                                device=device)
        dev = self.asm.device
        self.device = dev
        self.n_dofs = 3 * union.n_nodes
        self.dof_offsets_dev = torch.from_numpy(self.dof_offsets.astype(np.int64)).to(dev)
        counts = np.diff(self.dof_offsets)
        self.dof_instance = torch.from_numpy(np.repeat(np.arange(self.B, dtype=np.int64), counts)).to(dev)

    def concat(self, per_instance) -> torch.Tensor:
        """Per-instance DOF vectors -> one float64 device vector of the union."""
        a = np.concatenate([np.asarray(x, dtype=np.float64).reshape(-1) for x in per_instance])
        if a.size != self.n_dofs:
            raise ValueError(f"got {a.size} DOFs, the batch has {self.n_dofs}")
        return torch.from_numpy(a).to(self.device)

    def split(self, x: torch.Tensor) -> list[torch.Tensor]:
        o = self.dof_offsets
        return [x[int(o[i]):int(o[i + 1])] for i in range(self.B)]

    def segment_sumsq(self, x: torch.Tensor, out: torch.Tensor) -> torch.Tensor:
        check(lib().psx_segment_sumsq(self.B, ptr(self.dof_offsets_dev), ptr(x), ptr(out), _stream()),
              "psx_segment_sumsq")
        return out


@dataclass
class BatchedNewtonResult:
    u: list[torch.Tensor]
    converged: np.ndarray                 # (B,) bool
    steps_completed: np.ndarray           # (B,) int
    iterations: np.ndarray                # (n_steps, B) Newton iterations to convergence (0 = not)
    replays: int = 0
    residual_history: list = field(default_factory=list)  # per replay: (B,) ||R|| before the update


class BatchedNewton:
    def __init__(self, batch: MeshBatch, fixed_dofs, precision: str | None = None, pcg_iterations: int = 500,
                 pcg_rtol: float = 1e-8, preconditioner: str = "block-jacobi", use_graph: bool = True,
                 levels_per_aggregate: int = 4, per_instance_cg: bool = True):
        """``fixed_dofs``: per instance, its clamped DOFs in local numbering.
        ``preconditioner``: "none", "jacobi", "block-jacobi" or "two-level" (block-Jacobi
        plus rigid-body modes of slices of about ``levels_per_aggregate`` cross-sections).
        ``per_instance_cg``: run one CG per instance (own step lengths and residual test,
        ``psx_pcg_batched``) instead of one CG over the whole block-diagonal system; with
        the shared step lengths of the latter every instance converges at the rate of the
        worst-conditioned one (block-Jacobi and two-level; the plain Jacobi and
        unpreconditioned options always use one CG)."""
        self.batch = batch
        asm = batch.asm
        self.asm = asm
        self.precision = precision or asm.precision
        dev = asm.device
        n = batch.n_dofs
        self.n = n
        if len(fixed_dofs) != batch.B:
            raise ValueError("one fixed-DOF array per instance")
        mask = np.zeros(n, dtype=np.uint8)
        for i, fd in enumerate(fixed_dofs):
            mask[batch.dof_offsets[i] + np.asarray(fd, dtype=np.int64)] = 1
        self.fixed_u8 = torch.from_numpy(mask).to(dev)
        self.free = torch.from_numpy((mask == 0).astype(np.float64)).to(dev)
        self.pcg_iterations = int(pcg_iterations)
        self.pcg_rtol = float(pcg_rtol)
        # the batch's CSR has the assembler's node-blocked layout (PSX_PCG_NODAL)
        self.precond = {"none": _lib.PSX_PRECOND_NONE, "jacobi": _lib.PSX_PRECOND_JACOBI,
                        "block-jacobi": _lib.PSX_PRECOND_BJACOBI,
                        "two-level": _lib.PSX_PRECOND_BJACOBI}[preconditioner] | _lib.PSX_PCG_NODAL
        self.coarse = None
        if preconditioner == "two-level":
            from psierra_b200.coarse import CoarseSpace

            self.coarse = CoarseSpace(batch.mesh.nodes, batch.mesh.elements, mask, batch.node_offsets,
                                      levels_per_aggregate, device=dev)
        self.use_graph = use_graph
        f64 = dict(dtype=torch.float64, device=dev)
        B = batch.B
        self.u = torch.zeros(n, **f64)
        self.f = asm.new_f()
        self.k = asm.new_k(self.precision)
        self.f_step = torch.zeros(n, **f64)
        self.r = torch.zeros(n, **f64)
        self.rhs = torch.zeros(n, **f64)
        self.du = torch.zeros(n, **f64)
        self.scale = torch.ones(n, **f64)
        self.inv_scale = torch.ones(n, **f64)
        self.act_dof = torch.zeros(n, **f64)
        self.rn2 = torch.zeros(B, **f64)
        self.tol2 = torch.full((B,), float("inf"), **f64)
        self.act_b = torch.zeros(B, dtype=torch.bool, device=dev)
        self.act_f = torch.zeros(B, **f64)
        self._zero = torch.zeros((), **f64)
        self.per_instance_cg = per_instance_cg and preconditioner in ("block-jacobi", "two-level")
        nb = ctypes.c_int64()
        if self.per_instance_cg:
            check(lib().psx_pcg_batched_work_bytes(n, B, ctypes.byref(nb)), "psx_pcg_batched_work_bytes")
            self.node_seg = torch.from_numpy(np.repeat(np.arange(B, dtype=np.int32),
                                                       np.diff(batch.node_offsets))).to(dev)
            self.seg_iters = torch.zeros(B, dtype=torch.int32, device=dev)
        else:
            check(lib().psx_pcg_work_bytes(n, self.precond, ctypes.byref(nb)), "psx_pcg_work_bytes")
        self.pcg_work = torch.empty(int(nb.value), dtype=torch.uint8, device=dev)
        self.pcg_status = torch.zeros((int(lib().psx_status_bytes()) + 3) // 4, dtype=torch.int32, device=dev)
        self._graph: torch.cuda.CUDAGraph | None = None

    # ------------------------------------------------------------------ one iteration
    def _body(self) -> None:
        asm, d = self.asm, self.asm.dev
        vp = _lib.PSX_FP64 if self.k.dtype == torch.float64 else _lib.PSX_FP32_MIXED
        asm.assemble(self.u, want_f=True, want_k=True, precision=self.precision, f_out=self.f, k_out=self.k,
                     check_status=False)
        check(lib().psx_csr_dirichlet(self.n, ptr(d["indptr"]), ptr(d["indices"]), ptr(self.k), vp,
                                      ptr(self.fixed_u8), _stream()), "psx_csr_dirichlet")
        torch.sub(self.f_step, self.f, out=self.r)
        self.r.mul_(self.free)
        self.batch.segment_sumsq(self.r, self.rn2)
        torch.ge(self.rn2, self.tol2, out=self.act_b)
        self.act_f.copy_(self.act_b)
        torch.index_select(self.act_f, 0, self.batch.dof_instance, out=self.act_dof)
        # inactive instances get an exactly zero right-hand side (a where, not a product: a
        # retired instance's residual may be NaN, and NaN * 0 would reach every instance
        # through the CG's shared step lengths)
        torch.mul(self.r, self.inv_scale, out=self.rhs)
        torch.where(self.act_dof > 0, self.rhs, self._zero, out=self.rhs)
        self.du.zero_()
        if self.coarse is not None:
            self.coarse.update(self.k, d["indptr"], d["indices"])
        if self.per_instance_cg:
            check(lib().psx_pcg_batched(self.n, ptr(d["indptr"]), ptr(d["indices"]), ptr(self.k), vp, ptr(self.rhs),
                                        ptr(self.du), self.pcg_rtol, 0.0, self.pcg_iterations, self.precond,
                                        self.batch.B, ptr(self.batch.dof_offsets_dev), ptr(self.node_seg),
                                        self.coarse.struct_ptr() if self.coarse is not None else None,
                                        ptr(self.pcg_work), self.pcg_work.numel(), ptr(self.pcg_status),
                                        ptr(self.seg_iters), _stream()), "psx_pcg_batched")
        elif self.coarse is not None:
            check(lib().psx_pcg_coarse(self.n, ptr(d["indptr"]), ptr(d["indices"]), ptr(self.k), vp, ptr(self.rhs),
                                       ptr(self.du), self.pcg_rtol, 0.0, self.pcg_iterations, self.precond,
                                       self.coarse.struct_ptr(), ptr(self.pcg_work), self.pcg_work.numel(),
                                       ptr(self.pcg_status), _stream(), 0), "psx_pcg_coarse")
        else:
            check(lib().psx_pcg_enqueue(self.n, ptr(d["indptr"]), ptr(d["indices"]), ptr(self.k), vp, ptr(self.rhs),
                                        ptr(self.du), self.pcg_rtol, 0.0, self.pcg_iterations, self.precond,
                                        ptr(self.pcg_work), self.pcg_work.numel(), ptr(self.pcg_status), _stream()),
                  "psx_pcg_enqueue")
        self.du.mul_(self.scale)
        self.u.add_(self.du)

    def _capture(self) -> None:
        # warm up once eagerly with every instance inactive (u unchanged), then capture
        saved = self.tol2.clone()
        self.tol2.fill_(float("inf"))
        s = torch.cuda.Stream(device=self.asm.device)
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            self._body()
        torch.cuda.current_stream().wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self._body()
        torch.cuda.synchronize()
        self.tol2.copy_(saved)
        self._graph = g

    def iterate(self) -> None:
        """One Newton iteration of every active instance (a graph replay)."""
        if self.use_graph:
            if self._graph is None:
                self._capture()
            self._graph.replay()
        else:
            self._body()

    # ------------------------------------------------------------------ driver
    def solve(self, f_ext: torch.Tensor, n_steps: int = 8, nr_iterations: int = 25,
              nr_tol: float = 1e-8, max_halvings: int = 16, max_growth: float = 100.0) -> BatchedNewtonResult:
        """Incremental Newton of every instance with full steps and a divergence guard:
        a trial point is rejected, and its step length alpha halved, when its residual is
        non-finite (an inverted element) or more than ``max_growth`` times the residual
        at the last accepted point.  (The reference's line search, analysis/line_search.py:
        120-260, also rejects moderate growth; measured on the 256-beam batch that cuts the
        steps of instances that converge quadratically after one larger residual: 175 of
        256 converged in 585 replays, against 256 with this guard.)  Every trial is one
        replay; an instance gives up after ``max_halvings`` halvings of one step or
        ``nr_iterations`` accepted Newton iterations, and is then retired at its last
        converged load step."""
        b = self.batch
        B = b.B
        dev = self.asm.device
        f_ext = f_ext.to(dev, torch.float64)
        counts = np.diff(b.dof_offsets)
        dofs = lambda mask: torch.from_numpy(np.repeat(mask, counts)).to(dev)  # noqa: E731
        self.u.zero_()
        u_acc = self.u.clone()
        direction = torch.zeros_like(self.u)  # each instance's Newton step from its accepted point
        alive = np.ones(B, dtype=bool)
        steps_done = np.zeros(B, dtype=np.int64)
        its = np.zeros((n_steps, B), dtype=np.int64)
        hist = []
        replays = 0
        fn2 = torch.zeros(B, dtype=torch.float64, device=dev)
        if self.use_graph and self._graph is None:
            self._capture()
        for step in range(1, n_steps + 1):
            lam = step / n_steps
            torch.mul(f_ext, lam, out=self.f_step)
            b.segment_sumsq(self.f_step * self.free, fn2)
            fn = np.sqrt(fn2.cpu().numpy())
            ref = np.where(fn >= 1e-12, fn, 1.0)
            tol = nr_tol * ref
            self.tol2.copy_(torch.from_numpy(np.where(alive, tol * tol, np.inf)))
            torch.index_select(torch.from_numpy(ref).to(dev), 0, b.dof_instance, out=self.scale)
            torch.reciprocal(self.scale, out=self.inv_scale)
            conv = ~alive  # retired instances take no part
            accepted = np.zeros(B, dtype=np.int64)  # accepted points (the start counts)
            rn_acc = np.full(B, np.inf)  # residual at the last accepted point
            alpha = np.ones(B)
            direction.zero_()
            for _ in range(4 * nr_iterations):
                self.iterate()
                replays += 1
                rn = np.sqrt(self.rn2.cpu().numpy())
                # the replay assembled with check_status=False: a bounded wait that gave
                # up leaves a K_T summed out of order, so no instance may use this step
                raise_if_wait_gave_up(self.asm.status_counts()[3])
                hist.append(rn)
                active = alive & ~conv
                with np.errstate(invalid="ignore"):
                    ok = np.isfinite(rn) & ((accepted == 0) | (rn < tol) | (rn <= max_growth * rn_acc))
                acc = active & ok
                rej = active & ~ok
                accepted[acc] += 1
                rn_acc[acc] = rn[acc]
                alpha[acc] = 1.0
                newly = acc & (rn < tol)  # the device's test (it gave them no step)
                its[step - 1, newly] = accepted[newly]
                # the replay also took a full step from every trial point: the accepted
                # ones keep it as their new direction; the rejected ones go back from
                # their trial point (accepted point + alpha direction) to alpha / 2
                if rej.any():
                    m = dofs(rej)
                    back = torch.where(m, self.du + (0.5 * torch.from_numpy(np.repeat(alpha, counts)).to(dev)) * direction,
                                       self._zero)
                    self.u.sub_(back)
                    alpha[rej] *= 0.5
                torch.where(dofs(acc), self.du, direction, out=direction)
                bad = (rej & (alpha < 0.5 ** max_halvings)) | (active & (accepted > nr_iterations) & ~newly)
                alive &= ~bad
                conv |= newly | bad
                if bad.any():
                    # back to its last converged state: a non-finite u would make its
                    # tangent block non-finite
                    torch.where(dofs(bad), u_acc, self.u, out=self.u)
                if conv.all():
                    break
                # freeze the instances that are done
                self.tol2.copy_(torch.from_numpy(np.where(conv, np.inf, tol * tol)))
            alive &= conv  # not converged: retired at its last step
            keep = dofs(alive)
            u_acc = torch.where(keep, self.u, u_acc)
            self.u.copy_(u_acc)
            steps_done[alive] = step
        return BatchedNewtonResult(b.split(u_acc), alive.copy(), steps_done, its, replays, hist)
