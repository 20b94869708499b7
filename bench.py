"""Benchmark of the Tet4 Total-Lagrangian NeoHookean f_int + K_T assembly (one B200 per rank).

Workload (the configuration the headline metric is quoted on): unit cube, 80^3 hex
cells x 6 = 3,072,000 Tet4, 531,441 nodes, NeoHookean E = 3 kPa, nu = 0.45, seeded
displacement 0.05 sin(pi x) sin(pi y) z e_z + U(-1e-4, 1e-4).  One step = one fused
f_int + K_T assembly into the fixed CSR pattern (70,336,089 values) with inputs
resident in HBM.  The K values (281 MB FP32, 563 MB FP64) exceed the 126 MB L2, so
every step streams its outputs to HBM.

Reported: elements/s of the FP32-mixed path (``value``), the FP64 path beside it,
the error of the mixed tangent against the FP64 one, the roofline of the kernel
(algorithmic bytes / CUDA-event time vs the measured HBM copy bandwidth), the
end-to-end rate through the drop-in element API with host buffers, and the
reference CPU path (the numpy restatement of pSierra's element loop + COO->CSR)
timed on this host's cores.

``--impl reference`` times only that CPU path.  Multi-GPU: replicas only (each
rank assembles its own copy; no collective on the data path).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Tet4 f_int+K_T elems/s and K·v HBM GB/s, FP32-mixed vs FP64 at ≤1e-6 rel"
def workload(cells: int, elements: int, nodes: int) -> str:
    """The workload line of ``config``: the cube of ``cells``^3 Kuhn cells (80 by default)."""
    return (f"cube {cells}^3 Kuhn Tet4 ({elements:,} elements, {nodes:,} nodes), NeoHookean E=3e3 nu=0.45, "
            "u=0.05 sin(pi x) sin(pi y) z e_z + U(+-1e-4); one fused f_int+K_T assembly per step")


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one launch, from one ncu
# capture of the FP32-mixed f+K and K.v launches on the cube 56^3 (1,053,696 elements);
# the traffic grows with the element count, so it is scaled by E for this workload.
NCU_CAPTURE_ELEMENTS = 1053696
NCU_TRAFFIC = {"fk32": 98.47552e6 + 102.580736e6, "kv32": 52.138752e6 + 1.884416e6}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cells", type=int, default=80, help="cube cells per side (80 = the headline workload)")
    ap.add_argument("--cpu-sample", type=int, default=40000, help="elements in the bounded CPU sample")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline (profiling runs)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-tet10", action="store_true", help="skip the Tet10 assembly measurement")
    ap.add_argument("--no-fbar", action="store_true", help="skip the Tet4Fbar assembly measurement")
    ap.add_argument("--no-pcg", action="store_true", help="skip the PCG iteration measurement")
    ap.add_argument("--no-oracle", action="store_true", help="skip the accuracy check against the oracle")
    ap.add_argument("--dr-iterations", type=int, default=1000,
                    help="fused dynamic-relaxation pseudo-steps timed per precision (0 = skip)")
    ap.add_argument("--oracle-nodes", type=int, default=2000, help="nodes whose rows the oracle checks")
    return ap.parse_args()


def make_problem(cells: int):
    from psierra_b200 import meshgen
    from psierra_b200.material import IsotropicElasticParameters, NeoHookean

    m = meshgen.box_tet4(1.0, 1.0, 1.0, cells, cells, cells)
    u = meshgen.cube_smooth_u(m, seed=2024)
    p = IsotropicElasticParameters()
    p.set_from_youngs_poisson(youngs_modulus=3e3, poissons_ratio=0.45, mass_density=1000.0)
    return m, u, NeoHookean(p)


# --------------------------------------------------------------------------- CPU baseline
def _cpu_chunk(args):
    from oracle.assembly import element_loop

    X, els, u, mu, kappa = args
    t = time.perf_counter()
    kl, fl = element_loop(X, els, u, mu, kappa)  # assemble_internal_forces sweep
    kl, fl = element_loop(X, els, u, mu, kappa)  # assemble_tangent_stiffness_matrix sweep
    return time.perf_counter() - t, kl, fl


def cpu_baseline(m, u, mat, sample: int):
    """Reference algorithm (two element sweeps + COO->CSR + np.add.at) on a bounded sample."""
    import multiprocessing as mp

    from oracle.assembly import assemble_sparse, assemble_vector, coo_indices, element_dofs

    cores = os.cpu_count() or 1
    sample = min(sample, m.n_elements)
    rng = np.random.default_rng(0)
    start = int(rng.integers(0, m.n_elements - sample + 1))
    els = m.elements[start:start + sample]
    mu, kappa = mat.parameters.shear_modulus, mat.parameters.bulk_modulus
    chunks = np.array_split(np.arange(sample), cores)
    # each worker gets only the nodes its elements use (renumbered locally): the
    # per-element arithmetic is unchanged, and the timed map does not ship the whole
    # mesh to every process
    jobs = []
    for c in chunks:
        if c.size:
            used, local = np.unique(els[c], return_inverse=True)
            jobs.append((m.nodes[used], local.reshape(els[c].shape), u[used], mu, kappa))
    ctx = mp.get_context("spawn")
    with ctx.Pool(len(jobs)) as pool:
        pool.map(_cpu_chunk, [(m.nodes, els[:8], u, mu, kappa)] * len(jobs))  # warm the workers
        t0 = time.perf_counter()
        res = pool.map(_cpu_chunk, jobs)
        t_loop = time.perf_counter() - t0
    kl = np.concatenate([r[1] for r in res])
    fl = np.concatenate([r[2] for r in res])
    t1 = time.perf_counter()
    ed = element_dofs(els)
    r, c = coo_indices(ed)
    assemble_vector(fl, ed, m.n_dofs)
    assemble_sparse(kl, r, c, m.n_dofs)
    t_asm = time.perf_counter() - t1
    total = t_loop + t_asm
    return {
        "value": sample / total,
        "unit": "elements/s",
        "cores": len(jobs),
        "kind": "port",
        "sample": (f"{sample} contiguous elements of the workload mesh: the reference's two element sweeps "
                   f"(assemble_internal_forces + assemble_tangent_stiffness_matrix) split over {len(jobs)} "
                   f"processes ({t_loop:.2f} s), then COO->CSR + np.add.at in one process ({t_asm:.2f} s)"),
    }


def oracle_rows_check(m, u, mat, asm, k64, f64, k32, f32, count: int = 2000, seed: int = 17):
    """Accuracy of both GPU results against the oracle (the checker, outside any timed
    region): the rows of ``count`` seeded nodes, which the elements incident to them give
    exactly (``oracle.sample``)."""
    from oracle import sample as osample

    t0 = time.perf_counter()
    nodes = osample.sample_nodes(m.n_nodes, count, seed)
    dofs, K_ref, f_ref = osample.sampled_rows(m.nodes, m.elements, u, mat.parameters.shear_modulus,
                                              mat.parameters.bulk_modulus, nodes)
    out = {}
    ip, ix = asm.pattern.indptr, asm.pattern.indices
    for tag, k, f in (("fp64", k64, f64), ("mixed", k32, f32)):
        same, err = osample.compare_rows(osample.gpu_rows(ip, ix, k.double().cpu().numpy(), dofs), K_ref)
        fd = f.cpu().numpy()[dofs]
        out[f"K_{tag}_vs_oracle_max_rel"] = err
        out[f"f_{tag}_vs_oracle_rel2"] = float(np.linalg.norm(fd - f_ref) / np.linalg.norm(f_ref))
        out[f"pattern_{tag}_equal_oracle"] = bool(same)
    out["oracle_sample"] = (f"rows of {nodes.size} seeded nodes ({dofs.size} DOFs, {K_ref.nnz} K values): "
                            f"the oracle evaluates the elements incident to them and sums them by COO->CSR "
                            f"({time.perf_counter() - t0:.1f} s)")
    return out


# --------------------------------------------------------------------------- clocks
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        self.proc.wait(timeout=10)
        rows = [ln.split(",") for ln in open(self.path).read().strip().splitlines() if ln.strip()]
        os.unlink(self.path)
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].strip().replace(".", "").isdigit()]
        if not sm:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[j] for r in rows if len(r) >= 9 for j in range(4) if "Active" in r[5 + j]
                          and "Not" not in r[5 + j]})
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(rows[0][2]), "samples": len(sm),
                "reasons": reasons}


# --------------------------------------------------------------------------- GPU timing
def time_steps(fn, steps: int, warmup: int, sync_all):
    import torch

    for _ in range(warmup):
        fn()
    # keep warming until the clocks have ramped (at least 0.5 s of work)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < 0.5:
        fn()
        torch.cuda.synchronize()
    sync_all()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    start.record()
    for _ in range(steps):
        fn()
    end.record()
    torch.cuda.synchronize()
    return start.elapsed_time(end) / steps  # ms per step


def time_steps_flushed(fn, steps: int, warmup: int, sync_all, flush):
    """Like ``time_steps`` for a working set that fits in L2: ``flush`` (a write larger
    than L2) runs before every step, outside the per-step event pair."""
    import torch

    for _ in range(warmup):
        flush()
        fn()
    sync_all()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for a, b in ev:
        flush()
        a.record()
        fn()
        b.record()
    torch.cuda.synchronize()
    return sum(a.elapsed_time(b) for a, b in ev) / steps


def dr_benchmark(asm, k_vals, u_dev, m, iterations: int, sync_all, cells: int = 80):
    """The workload's dynamic relaxation: ``iterations`` fused matrix-free pseudo-steps
    (K_T(u) x on the fly, the viscous update of psierra analysis/dynamic_relaxation.py:
    296-299, 378-382 with damping c = 0.1, dt = 1), per precision, on the cube clamped at
    z = 0 with the reference's Gerschgorin lumped mass (dynamic_relaxation.py:87-128,
    safety factor 1.1) built from the assembled tangent.  One launch per pseudo-step; the
    working set (connectivity, X, u and five DOF vectors, ~150 MB) exceeds the L2."""
    import torch

    dev = u_dev.device
    n = 3 * m.n_nodes
    indptr = torch.from_numpy(asm.pattern.indptr.astype(np.int64)).to(dev)
    rows = torch.repeat_interleave(torch.arange(n, device=dev), indptr[1:] - indptr[:-1])
    row = torch.zeros(n, dtype=torch.float64, device=dev).index_add_(0, rows, k_vals.abs().double())
    del rows
    dt, sf, c = 1.0, 1.1, 0.1
    mdiag = 0.25 * sf * dt * dt * torch.clamp(row, min=1e-6 * float(row.max()))
    minv = 1.0 / mdiag
    zfix = np.flatnonzero(np.isclose(m.nodes[:, 2], 0.0))
    minv[torch.from_numpy(np.concatenate([3 * zfix + k for k in range(3)])).to(dev)] = 0.0
    c1, c2 = (2 - c * dt) / (2 + c * dt), 2 * dt / (2 + c * dt)
    b = torch.from_numpy(np.random.default_rng(5).standard_normal(n)).to(dev)
    b.mul_(minv != 0)
    x = torch.zeros(n, dtype=torch.float64, device=dev)
    vel = torch.zeros_like(x)
    E, N = m.n_elements, m.n_nodes
    # conn, X, u; x read, b, 1/m, vel read + write, x write
    bytes_it = 16 * E + 48 * N + 24 * N * 6
    out = {"workload": f"cube {cells}^3 clamped at z = 0, Gerschgorin lumped mass (sf 1.1), damping 0.1, dt 1; "
                       f"{iterations} fused K(u)-matrix-free pseudo-steps (psx_tet4_dr_step) per precision",
           "iterations": iterations, "algorithmic_bytes_per_iteration": bytes_it}
    for prec in ("fp32-mixed", "fp64"):
        x.zero_()
        vel.zero_()
        for _ in range(5):
            asm.dr_step(u_dev, b, minv, x, vel, c1, c2, dt, precision=prec, check_status=False)
        x.zero_()
        vel.zero_()
        sync_all()
        a = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(iterations):
            asm.dr_step(u_dev, b, minv, x, vel, c1, c2, dt, precision=prec, check_status=False)
        e.record()
        torch.cuda.synchronize()
        asm.raise_on_bad_elements(u_dev)
        ms = a.elapsed_time(e)
        r = b - asm.kv(u_dev, x, precision="fp64")
        out[prec.replace("-", "_")] = {
            "ms_total": ms, "ms_per_iteration": ms / iterations, "gbs": bytes_it * iterations / (ms * 1e-3) / 1e9,
            "relative_residual_after": float((r * (minv != 0)).norm() / b.norm())}
    return out


# FP64 floating-point work of the FP64 f+K element sweep, per element: 2 x DFMA + DADD + DMUL
# thread instructions of tet4_persistent_kernel<double, F|K> from the ncu counters
# smsp__sass_thread_inst_executed_op_d{fma,add,mul}_pred_on.sum of one launch on the 56^3
# cube (467.8M, 207.6M, 250.8M for 1,053,696 elements).
FP64_FLOPS_PER_ELEMENT = (2 * 467841024 + 207578112 + 250779648) / 1053696


def fp64_compute_roofline(E, ms, roofs):
    """The FP64 sweep against its compute roof (FP64 FLOPs / time vs the FMA roof)."""
    if FP64_FLOPS_PER_ELEMENT is None:
        return {}
    tf = FP64_FLOPS_PER_ELEMENT * E / (ms * 1e-3) / 1e12
    return {"fp64_flops_per_element": FP64_FLOPS_PER_ELEMENT, "fp64_tflops": tf,
            "fp64_compute_frac": tf / roofs["fp64_tflops"]}


def compute_roofs(dev, iters: int = 40000, reps: int = 5):
    """FP64 and FP32 CUDA-core FMA throughput of this GPU (TFLOP/s), measured with the
    library's FMA kernel (psx_fma_roof): 8 resident blocks of 256 threads per SM, 8
    independent FMA chains per thread, CUDA events around the launches."""
    import ctypes

    import torch

    from psierra_b200 import _lib

    L = _lib.lib()
    blocks = 8 * torch.cuda.get_device_properties(dev).multi_processor_count
    sink = torch.empty(int(L.psx_fma_roof_sink_bytes(blocks)), dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    out = {}
    for name, prec in (("fp64", _lib.PSX_FP64), ("fp32", _lib.PSX_FP32_MIXED)):
        flops = ctypes.c_double()
        for _ in range(2):
            _lib.check(L.psx_fma_roof(prec, iters, blocks, _lib.ptr(sink), ctypes.byref(flops), stream), "psx_fma_roof")
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            _lib.check(L.psx_fma_roof(prec, iters, blocks, _lib.ptr(sink), ctypes.byref(flops), stream), "psx_fma_roof")
        b.record()
        torch.cuda.synchronize()
        out[f"{name}_tflops"] = flops.value * reps / (a.elapsed_time(b) * 1e-3) / 1e12
    out["method"] = (f"psx_fma_roof: {blocks} blocks x 256 threads, 8 independent FMA chains x {iters} steps per "
                     f"thread, {reps} launches timed with CUDA events")
    return out


def peak_hbm():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        m, u, mat = make_problem(args.cells)
        vals = []
        for i in range(args.warmup + args.steps):
            cb = cpu_baseline(m, u, mat, args.cpu_sample)  # the sample size of the other arm's baseline
            if i >= args.warmup:
                vals.append(cb["value"])
        v = float(np.median(vals))
        cb["value"] = v
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": v, "unit": "elements/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * m.n_elements / v,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload(args.cells, m.n_elements, m.n_nodes), "elements": m.n_elements,
                       "nodes": m.n_nodes},
            "cpu_baseline": cb, "e2e": {"value": v, "unit": "elements/s", "h2d_bytes_per_step": 0,
                                        "d2h_bytes_per_step": 0}}))
        return

    import torch

    if world > 1:
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    dev = torch.device("cuda", torch.cuda.current_device())

    def sync_all():
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    m, u, mat = make_problem(args.cells)
    cb = None
    if rank == 0 and not args.no_cpu:
        cb = cpu_baseline(m, u, mat, args.cpu_sample)

    from psierra_b200.assembler import GPUAssembler
    from psierra_b200.element import Tet4TotalLagrangian

    asm = GPUAssembler(m.nodes, m.elements, mat, precision="fp32-mixed", device=dev)
    u_dev = torch.from_numpy(u.reshape(-1)).to(dev)
    f32 = asm.new_f()
    k32 = asm.new_k("fp32-mixed")
    f64 = asm.new_f()
    k64 = asm.new_k("fp64")
    E, N, nnz = m.n_elements, m.n_nodes, asm.nnz

    # correctness of the timed configuration (and the mixed-vs-FP64 error)
    asm.assemble(u_dev, precision="fp64", f_out=f64, k_out=k64)
    asm.assemble(u_dev, precision="fp32-mixed", f_out=f32, k_out=k32)
    k_err = float(((k32.double() - k64).abs().max() / k64.abs().max()).item())
    f_err = float(((f32 - f64).norm() / f64.norm()).item())
    accuracy = {"K_mixed_vs_fp64_max_rel": k_err, "f_mixed_vs_fp64_rel2": f_err}
    if rank == 0 and not args.no_oracle:
        accuracy.update(oracle_rows_check(m, u, mat, asm, k64, f64, k32, f32, count=args.oracle_nodes))

    def step_mixed():
        asm.assemble(u_dev, precision="fp32-mixed", f_out=f32, k_out=k32, check_status=False)

    def step_fp64():
        asm.assemble(u_dev, precision="fp64", f_out=f64, k_out=k64, check_status=False)

    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    ms_mixed = time_steps(step_mixed, args.steps, args.warmup, sync_all)
    clk = clocks.stop()
    ms_fp64 = time_steps(step_fp64, args.steps, args.warmup, sync_all)
    asm.raise_on_bad_elements(u_dev)

    # matrix-free K_T(u) v (the dynamic-relaxation product): reads conn, X, u, v; writes y
    v_dev = torch.from_numpy(np.random.default_rng(7).standard_normal(3 * N)).to(dev)
    y32 = asm.new_f()
    y64 = asm.new_f()
    asm.kv(u_dev, v_dev, precision="fp64", y_out=y64)
    asm.kv(u_dev, v_dev, precision="fp32-mixed", y_out=y32)
    kv_err = float(((y32 - y64).norm() / y64.norm()).item())
    # its working set (~100 MB at 3M elements) fits in L2: flush a 512 MB buffer before each step
    scrub = torch.empty(512 << 20, dtype=torch.uint8, device=dev)
    flush = lambda: scrub.fill_(1)  # noqa: E731
    ms_kv32 = time_steps_flushed(lambda: asm.kv(u_dev, v_dev, precision="fp32-mixed", y_out=y32, check_status=False),
                                 args.steps, args.warmup, sync_all, flush)
    ms_kv64 = time_steps_flushed(lambda: asm.kv(u_dev, v_dev, precision="fp64", y_out=y64, check_status=False),
                                 args.steps, args.warmup, sync_all, flush)
    del scrub

    dr = None
    if args.dr_iterations > 0:
        dr = dr_benchmark(asm, k32, u_dev, m, args.dr_iterations, sync_all, cells=args.cells)

    if world > 1:
        t = torch.tensor([ms_mixed, ms_fp64], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms_mixed, ms_fp64 = (float(x) for x in t.tolist())
        t = torch.tensor([ms_kv32, ms_kv64], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms_kv32, ms_kv64 = (float(x) for x in t.tolist())

    # PCG on the workload's FP32-mixed tangent, clamped at z = 0 (SPD): block-Jacobi,
    # a fixed number of iterations (rtol = atol = 0).  Time per iteration = difference of
    # two iteration counts (the set-up and the initial residual cancel).
    pcg = None
    if not args.no_pcg:
        import ctypes

        from psierra_b200 import _lib

        L = _lib.lib()
        n = 3 * N
        d = asm.dev
        kc = k32.clone()
        fixed = torch.zeros(n, dtype=torch.uint8, device=dev)
        zfix = np.flatnonzero(np.isclose(m.nodes[:, 2], 0.0))
        fixed[torch.from_numpy(np.concatenate([3 * zfix + c for c in range(3)])).to(dev)] = 1
        _lib.check(L.psx_csr_dirichlet(n, _lib.ptr(d["indptr"]), _lib.ptr(d["indices"]), _lib.ptr(kc),
                                       _lib.PSX_FP32_MIXED, _lib.ptr(fixed),
                                       torch.cuda.current_stream().cuda_stream), "psx_csr_dirichlet")
        rhs = torch.from_numpy(np.random.default_rng(11).standard_normal(n)).to(dev)
        xs = torch.zeros(n, dtype=torch.float64, device=dev)
        nb = ctypes.c_int64()
        _lib.check(L.psx_pcg_work_bytes(n, _lib.PSX_PRECOND_BJACOBI, ctypes.byref(nb)), "psx_pcg_work_bytes")
        pw = torch.empty(int(nb.value), dtype=torch.uint8, device=dev)
        pst = torch.zeros(16, dtype=torch.int32, device=dev)

        def run_pcg(iters, flags):
            xs.zero_()
            pst.zero_()
            _lib.check(L.psx_pcg_enqueue(n, _lib.ptr(d["indptr"]), _lib.ptr(d["indices"]), _lib.ptr(kc),
                                         _lib.PSX_FP32_MIXED, _lib.ptr(rhs), _lib.ptr(xs), 0.0, 0.0, iters,
                                         _lib.PSX_PRECOND_BJACOBI | flags, _lib.ptr(pw), pw.numel(), _lib.ptr(pst),
                                         torch.cuda.current_stream().cuda_stream), "psx_pcg_enqueue")

        def ms_per_iteration(flags, lo=10, hi=60):
            ms_lo = time_steps(lambda: run_pcg(lo, flags), max(1, args.steps // 2), args.warmup, sync_all)
            ms_hi = time_steps(lambda: run_pcg(hi, flags), max(1, args.steps // 2), args.warmup, sync_all)
            ms = (ms_hi - ms_lo) / (hi - lo)
            if world > 1:
                t = torch.tensor([ms], device=dev)
                torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
                ms = float(t.item())
            return ms

        ms_it = ms_per_iteration(_lib.PSX_PCG_NODAL)
        ms_row = ms_per_iteration(0)
        # Bytes the node-blocked format must move per iteration: the FP32 values once, one
        # column index per 3x3 block (nnz / 9: the three rows of a node share their column
        # list), and ~10 vectors of n doubles (p, q, x, r, z and the 3x3 preconditioner
        # blocks, 3 n).  The row-wise CSR equivalent (a column index per value) is beside it.
        bytes_it = 4 * nnz + 4 * (nnz // 9) + 8 * 10 * n
        bytes_csr = 8 * nnz + 8 * 10 * n
        pcg = {"workload": "block-Jacobi PCG on the FP32-mixed tangent of the same mesh, clamped at z = 0, "
                           "fixed iteration count, node-blocked SpMV (PSX_PCG_NODAL)", "ms_per_iteration": ms_it,
               "algorithmic_bytes_per_iteration": bytes_it, "gbs": bytes_it / (ms_it * 1e-3) / 1e9,
               "bytes_note": "frac is on the node-blocked bytes (values + nnz/9 indices + vectors); "
                             "csr_equivalent_frac charges a column index per value",
               "csr_equivalent_bytes_per_iteration": bytes_csr,
               "csr_equivalent_gbs": bytes_csr / (ms_it * 1e-3) / 1e9,
               "kernels_per_iteration": 3, "row_spmv_ms_per_iteration": ms_row}
        del kc, pw

    # algorithmic bytes per launch (conn 16 E + X,u 48 N + K nnz*s + f 24 N)
    bytes_mixed = 16 * E + 48 * N + 4 * nnz + 24 * N
    bytes_fp64 = 16 * E + 48 * N + 8 * nnz + 24 * N
    bytes_kv = 16 * E + 96 * N
    peak, peak_kind = peak_hbm()
    roofs = compute_roofs(dev)
    if pcg is not None:
        pcg["frac"] = pcg["gbs"] / peak
        pcg["csr_equivalent_frac"] = pcg["csr_equivalent_gbs"] / peak
    if dr is not None:
        for v in dr.values():
            if isinstance(v, dict) and "gbs" in v:
                v["frac"] = v["gbs"] / peak
    ach = bytes_mixed / (ms_mixed * 1e-3) / 1e9

    # Tet10: cube 30^3 Kuhn split upgraded to 10 nodes (162,000 elements, 226,981 nodes,
    # nnz 57,014,289), E = 1e4, nu = 0.4, seeded smooth displacement
    tet10 = None
    if not args.no_tet10:
        from psierra_b200 import meshgen
        from psierra_b200.material import IsotropicElasticParameters, NeoHookean

        m10 = meshgen.tet4_to_tet10(meshgen.box_tet4(1.0, 1.0, 1.0, 30, 30, 30))
        p10 = IsotropicElasticParameters()
        p10.set_from_youngs_poisson(youngs_modulus=1e4, poissons_ratio=0.4, mass_density=1000.0)
        a10 = GPUAssembler(m10.nodes, m10.elements, NeoHookean(p10), precision="fp32-mixed", device=dev)
        u10 = torch.from_numpy(meshgen.cube_smooth_u(m10, seed=7).reshape(-1)).to(dev)
        f10 = a10.new_f()
        k10s = a10.new_k("fp32-mixed")
        k10d = a10.new_k("fp64")
        a10.assemble(u10, precision="fp64", f_out=f10, k_out=k10d)
        a10.assemble(u10, precision="fp32-mixed", f_out=f10, k_out=k10s)
        err10 = float(((k10s.double() - k10d).abs().max() / k10d.abs().max()).item())
        ms10s = time_steps(lambda: a10.assemble(u10, precision="fp32-mixed", f_out=f10, k_out=k10s, check_status=False),
                           args.steps, args.warmup, sync_all)
        ms10d = time_steps(lambda: a10.assemble(u10, precision="fp64", f_out=f10, k_out=k10d, check_status=False),
                           args.steps, args.warmup, sync_all)
        if world > 1:
            t = torch.tensor([ms10s, ms10d], device=dev)
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            ms10s, ms10d = (float(x) for x in t.tolist())
        E10, N10, nnz10 = m10.n_elements, m10.n_nodes, a10.nnz
        b10s = 40 * E10 + 48 * N10 + 4 * nnz10 + 24 * N10
        b10d = 40 * E10 + 48 * N10 + 8 * nnz10 + 24 * N10
        tet10 = {"workload": "cube 30^3 Kuhn -> Tet10 (162,000 elements, 226,981 nodes, nnz 57,014,289), "
                             "E=1e4 nu=0.4, one fused f_int+K_T assembly",
                 "fp32_mixed": {"ms": ms10s, "elements_per_s": world * E10 / (ms10s * 1e-3),
                                "gbs": b10s / (ms10s * 1e-3) / 1e9, "frac": b10s / (ms10s * 1e-3) / 1e9 / peak_hbm()[0]},
                 "fp64": {"ms": ms10d, "elements_per_s": world * E10 / (ms10d * 1e-3),
                          "gbs": b10d / (ms10d * 1e-3) / 1e9, "frac": b10d / (ms10d * 1e-3) / 1e9 / peak_hbm()[0]},
                 "algorithmic_bytes_fp64": b10d, "K_mixed_vs_fp64_max_rel": err10}
        del a10, k10s, k10d

    # Tet4Fbar: cube 30^3 Kuhn (162,000 Tet4), E = 1e4, nu = 0.49, seeded smooth displacement;
    # f_int + tangent on the two-ring pattern (the reference's K_dev + K_vol)
    fbar = None
    if not args.no_fbar:
        from psierra_b200 import meshgen
        from psierra_b200.fbar import FbarAssembler
        from psierra_b200.material import IsotropicElasticParameters, NeoHookean

        mf = meshgen.box_tet4(1.0, 1.0, 1.0, 30, 30, 30)
        pf = IsotropicElasticParameters()
        pf.set_from_youngs_poisson(youngs_modulus=1e4, poissons_ratio=0.49, mass_density=1000.0)
        af = FbarAssembler(mf.nodes, mf.elements, NeoHookean(pf), device=dev)
        uf = torch.from_numpy(meshgen.cube_smooth_u(mf, seed=11).reshape(-1)).to(dev)
        af.assemble(uf)
        msf = time_steps(lambda: af.assemble(uf, check_status=False), args.steps, args.warmup, sync_all)
        if world > 1:
            t = torch.tensor([msf], device=dev)
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            msf = float(t.item())
        # conn, X and u, the two-ring K values (FP64) and f: what the sweep must move
        bytes_f = 16 * mf.n_elements + 48 * mf.n_nodes + 8 * af.nnz + 24 * mf.n_nodes
        fbar = {"workload": "cube 30^3 Kuhn Tet4Fbar (162,000 elements, 29,791 nodes), E=1e4 nu=0.49, "
                            "f_int + K_dev + K_vol on the two-ring pattern",
                "ms": msf, "elements_per_s": world * mf.n_elements / (msf * 1e-3), "nnz_two_ring": af.nnz,
                "algorithmic_bytes": bytes_f, "gbs": bytes_f / (msf * 1e-3) / 1e9,
                "frac": bytes_f / (msf * 1e-3) / 1e9 / peak_hbm()[0],
                "launches_per_call": 6}
        del af

    e2e = None
    if not args.no_e2e:
        el = Tet4TotalLagrangian(mat, precision="fp32-mixed", device=dev)
        el._setup(m)
        for _ in range(2):
            el.assemble_force_and_tangent(m, u)
        sync_all()
        t0 = time.perf_counter()
        n_e2e = max(2, min(args.steps, 5))
        for _ in range(n_e2e):
            el.assemble_force_and_tangent(m, u)
        torch.cuda.synchronize()
        dt = (time.perf_counter() - t0) / n_e2e
        # K values are widened to float64 on the device (the drop-in returns a float64 CSR,
        # like the reference), so each step downloads 8 bytes per value plus f
        e2e = {"value": world * E / dt, "unit": "elements/s", "h2d_bytes_per_step": 24 * N,
               "d2h_bytes_per_step": 24 * N + 8 * nnz,
               "path": "Tet4TotalLagrangian.assemble_force_and_tangent(mesh, u_host) -> (numpy f, scipy CSR)"}

    if rank == 0:
        from psierra_b200 import _lib

        split = asm.pattern.split and _lib.lib().psx_tet4_split_ready() == 1
        fk_kernel = ("tet4_split_kernel<float> F|K (per SM 8 element-tile warps + 8 owner-computes gather warps, "
                     "registers moved between them by setmaxnreg)" if split else
                     "tet4_persistent_kernel<float> F|K (element tiles + owner-computes gather in the same warps)")
        line = {
            "metric": METRIC, "value": world * E / (ms_mixed * 1e-3), "unit": "elements/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_mixed, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp32-mixed (K_T f32; f_int, det F, ln J f64)",
            "data": "synthetic",
            "config": {"workload": workload(args.cells, E, N), "elements": E, "nodes": N, "nnz": nnz,
                       "l2": (f"assembly: working set {'exceeds' if 4 * nnz > 126e6 else 'within'} L2 (K values "
                              f"{4 * nnz / 1e6:.0f} MB fp32 / {8 * nnz / 1e6:.0f} MB fp64 vs 126 MB L2); "
                              "K.v: 512 MB L2 flush before every timed step"),
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                         "traffic": NCU_TRAFFIC["fk32"] * E / NCU_CAPTURE_ELEMENTS,
                         "traffic_note": "bytes per launch: ncu DRAM read+write of the cube 56^3 launch scaled by "
                                         "elements (latency-bound: DRAM throughput 10.7% in that capture of the split kernel)",
                         "peak_kind": peak_kind,
                         "algorithmic_bytes_per_launch": bytes_mixed, "kernel": fk_kernel,
                         "launches_per_step": asm.launches_per_call("fp32-mixed")},
            "fp64": {"value": world * E / (ms_fp64 * 1e-3), "unit": "elements/s", "ms_per_step": ms_fp64,
                     "achieved_gbs": bytes_fp64 / (ms_fp64 * 1e-3) / 1e9,
                     "frac": bytes_fp64 / (ms_fp64 * 1e-3) / 1e9 / peak,
                     **fp64_compute_roofline(E, ms_fp64, roofs)},
            "compute_roofs": roofs,
            "mixed_over_fp64": ms_fp64 / ms_mixed,
            "kv": {"unit": "GB/s", "algorithmic_bytes_per_launch": bytes_kv,
                   "traffic": NCU_TRAFFIC["kv32"] * E / NCU_CAPTURE_ELEMENTS,
                   "fp32_mixed": {"ms": ms_kv32, "gbs": bytes_kv / (ms_kv32 * 1e-3) / 1e9,
                                  "frac": bytes_kv / (ms_kv32 * 1e-3) / 1e9 / peak,
                                  "elements_per_s": world * E / (ms_kv32 * 1e-3)},
                   "fp64": {"ms": ms_kv64, "gbs": bytes_kv / (ms_kv64 * 1e-3) / 1e9,
                            "frac": bytes_kv / (ms_kv64 * 1e-3) / 1e9 / peak,
                            "elements_per_s": world * E / (ms_kv64 * 1e-3)},
                   "mixed_vs_fp64_rel2": kv_err},
            "accuracy": accuracy,
            "tet10": tet10,
            "fbar": fbar,
            "pcg": pcg,
            "dynamic_relaxation": dr,
            "cpu_baseline": cb, "e2e": e2e, "gpu_launches": args.steps * asm.launches_per_call("fp32-mixed"),
            "gpu_launches_note": "assembly timed region; each K.v step is one launch as well",
            "clocks": clk,
        }
        print(json.dumps(line))
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
