"""Two-level preconditioner on the GPU: the coarse kernels against a dense restatement of
P, A_c = P^T K P assembled on the device, the two-level CG against block-Jacobi CG, and
the batched Newton with the coarse correction inside its CUDA graph."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from conftest import rel_2
from psierra_b200 import _lib, meshgen
from psierra_b200._lib import check, lib, ptr
from psierra_b200.assembler import GPUAssembler
from psierra_b200.batched import BatchedNewton, MeshBatch
from psierra_b200.coarse import CoarseSpace
from psierra_b200.material import NeoHookeanField
from test_batched_gpu import small_batch
from test_coarse import _dense_P

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda")


def _stream():
    return torch.cuda.current_stream().cuda_stream


def _two_beams(precision="fp64"):
    meshes = [meshgen.box_tet4(1.2, 0.1, 0.1, 48, 4, 4), meshgen.box_tet4(0.1, 0.8, 0.1, 4, 32, 4)]
    union, node_off, _ = meshgen.concat_meshes(meshes)
    mu, _, kappa = meshgen.lame_from_young_poisson(1e5, 0.3)
    asm = GPUAssembler(union.nodes, union.elements,
                       NeoHookeanField(np.full(union.n_elements, mu), np.full(union.n_elements, kappa)),
                       precision=precision)
    fixed = np.zeros(3 * union.n_nodes, dtype=np.uint8)
    for b, m in enumerate(meshes):
        axis = int(np.argmax(np.ptp(m.nodes, axis=0)))
        clamp = node_off[b] + meshgen.nodes_on_plane(m, axis, "min")
        fixed[np.concatenate([3 * clamp + c for c in range(3)])] = 1
    return meshes, union, node_off, asm, fixed


def _eliminated_tangent(asm, fixed, precision):
    u = torch.zeros(3 * asm.n_nodes, dtype=torch.float64, device=DEV)
    _, k = asm.assemble(u, want_f=False, want_k=True, precision=precision)
    d = asm.dev
    vp = _lib.PSX_FP64 if k.dtype == torch.float64 else _lib.PSX_FP32_MIXED
    check(lib().psx_csr_dirichlet(3 * asm.n_nodes, ptr(d["indptr"]), ptr(d["indices"]), ptr(k), vp,
                                  ptr(torch.from_numpy(fixed).to(DEV)), _stream()), "psx_csr_dirichlet")
    return k


def test_probe_and_restrict_kernels_match_dense_P():
    meshes, union, node_off, asm, fixed = _two_beams()
    cs = CoarseSpace(union.nodes, union.elements, fixed, node_off, levels_per_aggregate=4)
    P = _dense_P(union.nodes, cs.node_agg.cpu().numpy().astype(np.int64), fixed, cs.n_agg)
    colour = cs.agg_colour.cpu().numpy()
    v = torch.empty(3 * union.n_nodes, dtype=torch.float64, device=DEV)
    for c in range(cs.n_colours):
        for s in range(6):
            want = P[:, 6 * np.where(colour == c)[0] + s].sum(axis=1)
            got = cs.probe(c, s, v).cpu().numpy()
            assert np.abs(got - want).max() <= 1e-15 * max(1.0, np.abs(want).max())
    w = torch.randn(3 * union.n_nodes, dtype=torch.float64, device=DEV)
    out = torch.empty(6 * cs.n_agg, dtype=torch.float64, device=DEV)
    got = cs.restrict(w, out).cpu().numpy()
    want = P.T @ w.cpu().numpy()
    assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()


@pytest.mark.parametrize("precision", ["fp64", "fp32-mixed"])
def test_coarse_matrix_is_P_T_K_P(precision):
    import scipy.sparse as sp

    meshes, union, node_off, asm, fixed = _two_beams(precision)
    k = _eliminated_tangent(asm, fixed, precision)
    cs = CoarseSpace(union.nodes, union.elements, fixed, node_off, levels_per_aggregate=4)
    cs.update(k, asm.dev["indptr"], asm.dev["indices"])
    n = 3 * union.n_nodes
    K = sp.csr_matrix((k.double().cpu().numpy(), asm.pattern.indices, asm.pattern.indptr), shape=(n, n))
    P = _dense_P(union.nodes, cs.node_agg.cpu().numpy().astype(np.int64), fixed, cs.n_agg)
    Ac = P.T @ (K @ P)
    ba = cs.block_agg.cpu().numpy()
    for b in range(cs.n_blocks):
        sl = slice(6 * ba[b], 6 * ba[b + 1])
        m = 6 * (ba[b + 1] - ba[b])
        assert np.abs(cs.ac[b, :m, :m].cpu().numpy() - Ac[sl, sl]).max() <= 1e-11 * np.abs(Ac[sl, sl]).max()
    assert bool(cs.factor_ok.all())


def test_two_level_cg_matches_block_jacobi_in_far_fewer_iterations():
    meshes, union, node_off, asm, fixed = _two_beams()
    k = _eliminated_tangent(asm, fixed, "fp64")
    d = asm.dev
    n = 3 * union.n_nodes
    f = np.concatenate([meshgen.traction_nodal_forces(m, int(np.argmax(np.ptp(m.nodes, axis=0))), "max",
                                                      [0.0, 0.0, -10.0]) for m in meshes])
    b = torch.from_numpy(f * (fixed == 0)).to(DEV)
    cs = CoarseSpace(union.nodes, union.elements, fixed, node_off, levels_per_aggregate=4)
    cs.update(k, d["indptr"], d["indices"])
    prec = _lib.PSX_PRECOND_BJACOBI | _lib.PSX_PCG_NODAL
    nb = ctypes.c_int64()
    check(lib().psx_pcg_work_bytes(n, prec, ctypes.byref(nb)), "psx_pcg_work_bytes")
    work = torch.empty(int(nb.value), dtype=torch.uint8, device=DEV)
    st = torch.zeros((int(lib().psx_status_bytes()) + 3) // 4, dtype=torch.int32, device=DEV)
    out = {}
    for name in ("block-jacobi", "two-level"):
        x = torch.zeros(n, dtype=torch.float64, device=DEV)
        if name == "two-level":
            rc = lib().psx_pcg_coarse(n, ptr(d["indptr"]), ptr(d["indices"]), ptr(k), _lib.PSX_FP64, ptr(b), ptr(x),
                                      1e-10, 0.0, 100000, prec, cs.struct_ptr(), ptr(work), work.numel(), ptr(st),
                                      _stream(), 1)
        else:
            rc = lib().psx_pcg(n, ptr(d["indptr"]), ptr(d["indices"]), ptr(k), _lib.PSX_FP64, ptr(b), ptr(x), 1e-10,
                               0.0, 100000, prec, ptr(work), work.numel(), ptr(st), _stream())
        check(rc, name)
        s = st.cpu().numpy()
        assert s[5] == 0, (name, s)  # converged
        out[name] = (x.cpu().numpy(), int(s[4]))
    assert rel_2(out["two-level"][0], out["block-jacobi"][0]) < 1e-8
    assert out["two-level"][1] * 5 < out["block-jacobi"][1], out


def test_batched_newton_two_level_matches_block_jacobi():
    cases = small_batch(n=8, seed=5)
    mb = MeshBatch([c[0] for c in cases], [c[1] for c in cases], [c[2] for c in cases], precision="fp32-mixed")
    f = mb.concat([c[3] for c in cases])
    res = {}
    for name, its in (("block-jacobi", 3000), ("two-level", 300)):
        bn = BatchedNewton(mb, [c[4] for c in cases], pcg_iterations=its, pcg_rtol=1e-10, preconditioner=name,
                           levels_per_aggregate=2)
        res[name] = bn.solve(f, n_steps=3, nr_iterations=25, nr_tol=1e-8)
        assert res[name].converged.all(), name
    for a, b in zip(res["two-level"].u, res["block-jacobi"].u):
        assert rel_2(a.cpu().numpy(), b.cpu().numpy()) < 1e-6


@pytest.mark.parametrize("coarse,precision,nodal", [(False, "fp64", True), (True, "fp64", True),
                                                    (True, "fp32-mixed", True), (True, "fp64", False)])
def test_batched_cg_solves_each_instance_like_its_own_cg(coarse, precision, nodal):
    """psx_pcg_batched: one CG per segment of a block-diagonal system; each segment's
    solution equals that instance's own solve (psx_pcg, block-Jacobi) to the solver
    tolerance, and the segments converge with their own iteration counts (FP64 or FP32
    matrix values, node-blocked or row-wise SpMV)."""
    meshes, union, node_off, asm, fixed = _two_beams(precision)
    k = _eliminated_tangent(asm, fixed, precision)
    vp = _lib.PSX_FP64 if k.dtype == torch.float64 else _lib.PSX_FP32_MIXED
    d = asm.dev
    n = 3 * union.n_nodes
    f = np.concatenate([meshgen.traction_nodal_forces(m, int(np.argmax(np.ptp(m.nodes, axis=0))), "max",
                                                      [0.0, 0.0, -10.0 * (1 + 99 * b)]) for b, m in enumerate(meshes)])
    b = torch.from_numpy(f * (fixed == 0)).to(DEV)
    prec = _lib.PSX_PRECOND_BJACOBI | (_lib.PSX_PCG_NODAL if nodal else 0)
    B = len(meshes)
    seg_off = torch.from_numpy(3 * np.asarray(node_off, dtype=np.int64)).to(DEV)
    node_seg = torch.from_numpy(np.repeat(np.arange(B, dtype=np.int32), np.diff(node_off))).to(DEV)
    cs = None
    if coarse:
        cs = CoarseSpace(union.nodes, union.elements, fixed, node_off, levels_per_aggregate=4)
        cs.update(k, d["indptr"], d["indices"])
    nb = ctypes.c_int64()
    check(lib().psx_pcg_batched_work_bytes(n, B, ctypes.byref(nb)), "psx_pcg_batched_work_bytes")
    work = torch.empty(int(nb.value), dtype=torch.uint8, device=DEV)
    st = torch.zeros((int(lib().psx_status_bytes()) + 3) // 4, dtype=torch.int32, device=DEV)
    seg_iters = torch.zeros(B, dtype=torch.int32, device=DEV)
    x = torch.zeros(n, dtype=torch.float64, device=DEV)
    check(lib().psx_pcg_batched(n, ptr(d["indptr"]), ptr(d["indices"]), ptr(k), vp, ptr(b), ptr(x), 1e-12,
                                0.0, 20000, prec, B, ptr(seg_off), ptr(node_seg),
                                cs.struct_ptr() if cs is not None else None, ptr(work), work.numel(), ptr(st),
                                ptr(seg_iters), _stream()), "psx_pcg_batched")
    its = seg_iters.cpu().numpy()
    assert (its > 0).all() and st.cpu().numpy()[5] == 0, (its, st.cpu().numpy())
    # reference: each instance alone (block-Jacobi CG on its own block of the system)
    check(lib().psx_pcg_work_bytes(n, prec, ctypes.byref(nb)), "psx_pcg_work_bytes")
    work1 = torch.empty(int(nb.value), dtype=torch.uint8, device=DEV)
    for s in range(B):
        bs = torch.zeros_like(b)
        lo, hi = 3 * int(node_off[s]), 3 * int(node_off[s + 1])
        bs[lo:hi] = b[lo:hi]
        xs = torch.zeros_like(b)
        check(lib().psx_pcg(n, ptr(d["indptr"]), ptr(d["indices"]), ptr(k), vp, ptr(bs), ptr(xs), 1e-12,
                            0.0, 200000, prec, ptr(work1), work1.numel(), ptr(st), _stream()), "psx_pcg")
        assert st.cpu().numpy()[5] == 0
        assert rel_2(x[lo:hi].cpu().numpy(), xs[lo:hi].cpu().numpy()) < 1e-9, s


def test_device_newton_two_level_matches_block_jacobi():
    """DeviceNewton with the two-level preconditioner on a slender clamped beam: the same
    Newton iterations and displacement as block-Jacobi, in far fewer CG iterations."""
    from psierra_b200.newton import DeviceNewton

    m = meshgen.box_tet4(1.5, 0.1, 0.1, 60, 4, 4)
    mu, _, kappa = meshgen.lame_from_young_poisson(1e5, 0.3)
    f = torch.from_numpy(meshgen.traction_nodal_forces(m, 0, "max", [20.0, 0.0, -2.0])).to(DEV)
    clamp = meshgen.nodes_on_plane(m, 0, "min")
    fixed = np.concatenate([3 * clamp + c for c in range(3)])
    out = {}
    for pre in ("block-jacobi", "two-level"):
        asm = GPUAssembler(m.nodes, m.elements, NeoHookeanField(np.full(m.n_elements, mu), np.full(m.n_elements, kappa)))
        nt = DeviceNewton(asm, fixed, precision="fp64", pcg_tol=1e-12, pcg_maxiter=100000, preconditioner=pre)
        res = nt.solve(f, n_steps=2, nr_iterations=20, nr_tol=1e-10)
        assert res.converged, pre
        out[pre] = (res.u.cpu().numpy(), res.iteration_history, sum(res.pcg_iterations))
    assert out["two-level"][1] == out["block-jacobi"][1]
    assert rel_2(out["two-level"][0], out["block-jacobi"][0]) < 1e-9
    assert out["two-level"][2] * 4 < out["block-jacobi"][2], (out["two-level"][2], out["block-jacobi"][2])


def test_batched_cg_isolates_a_non_finite_instance():
    """A retired instance whose tangent block holds NaN (its displacement inverted
    elements) gets a zero right-hand side; the other instances' CGs, which share the
    launches but not the step lengths, must be unaffected: their solutions equal a solve
    with finite values everywhere, bit for bit."""
    meshes, union, node_off, asm, fixed = _two_beams()
    k = _eliminated_tangent(asm, fixed, "fp64")
    d = asm.dev
    n = 3 * union.n_nodes
    f = np.concatenate([meshgen.traction_nodal_forces(m, int(np.argmax(np.ptp(m.nodes, axis=0))), "max",
                                                      [0.0, 0.0, -10.0]) for m in meshes])
    b = torch.from_numpy(f * (fixed == 0)).to(DEV)
    lo0, hi0 = 0, 3 * int(node_off[1])
    b[lo0:hi0] = 0.0  # instance 0 retired
    prec = _lib.PSX_PRECOND_BJACOBI | _lib.PSX_PCG_NODAL
    B = len(meshes)
    seg_off = torch.from_numpy(3 * np.asarray(node_off, dtype=np.int64)).to(DEV)
    node_seg = torch.from_numpy(np.repeat(np.arange(B, dtype=np.int32), np.diff(node_off))).to(DEV)
    nb = ctypes.c_int64()
    check(lib().psx_pcg_batched_work_bytes(n, B, ctypes.byref(nb)), "psx_pcg_batched_work_bytes")
    work = torch.empty(int(nb.value), dtype=torch.uint8, device=DEV)
    st = torch.zeros((int(lib().psx_status_bytes()) + 3) // 4, dtype=torch.int32, device=DEV)
    indptr = d["indptr"].cpu().numpy()
    out = []
    for poison in (False, True):
        kk = k.clone()
        if poison:  # every value in the rows of instance 0
            kk[int(indptr[lo0]):int(indptr[hi0])] = float("nan")
        x = torch.zeros(n, dtype=torch.float64, device=DEV)
        check(lib().psx_pcg_batched(n, ptr(d["indptr"]), ptr(d["indices"]), ptr(kk), _lib.PSX_FP64, ptr(b), ptr(x),
                                    1e-10, 0.0, 5000, prec, B, ptr(seg_off), ptr(node_seg), None, ptr(work),
                                    work.numel(), ptr(st), None, _stream()), "psx_pcg_batched")
        out.append(x.clone())
    assert torch.equal(out[0][hi0:], out[1][hi0:])
    assert torch.isfinite(out[1][hi0:]).all() and out[1][hi0:].abs().max() > 0
