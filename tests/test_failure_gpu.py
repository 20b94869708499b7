"""Failure detection of the persistent assembly kernels (GPU), without a GPU fault.

Every wait of an element tile or a gather on another warp's progress is bounded: after
``wait_spins`` polls it gives up, sets status flag bit 0 and returns; every later wait of
the launch then returns at once, and the kernel runs to its end with every access in
bounds.  The host turns the flag into ``RuntimeError``.

These tests make a wait run out on purpose: they raise the gather-tile target of
granule 0 in the plan to a count no gather can reach, shrink the ring so that element
tiles must wait on that granule, and set a short wait limit.  The launch must return,
the flag must be set, the assembler must raise, and, with the plan restored, the next
call on the same context must give the bits of an untouched assembler.

NaN displacements: the reference tests only ``J <= 0.0``
(psierra ``element/tet4_total_lagrangian.py:110-112``), which is false for NaN, so a NaN
in u propagates into f_int and K_T of the elements that touch it and raises nothing.
The kernels behave the same way.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from psierra_b200 import meshgen
from psierra_b200.assembler import GPUAssembler
from psierra_b200.element import Tet4TotalLagrangian
from psierra_b200.material import IsotropicElasticParameters, NeoHookean

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda")
SHORT_WAIT = 2000  # polls: well under a millisecond with the kernels' 200 ns back-off


def _material(E=3e3, nu=0.45):
    p = IsotropicElasticParameters()
    p.set_from_youngs_poisson(youngs_modulus=E, poissons_ratio=nu, mass_density=1000.0)
    return NeoHookean(p)


def _cube(cells=24):
    m = meshgen.box_tet4(1.0, 1.0, 1.0, cells, cells, cells)
    u = meshgen.cube_smooth_u(m, seed=5)
    return m, torch.from_numpy(u.reshape(-1)).to(DEV)


def _small_ring(asm):
    # ring = next power of two >= span + lag + slack (16 granules on the 24^3 cube, which
    # has 21): element tiles of granules >= 16 wait for the gathers of granules >= 0
    asm.set_queue(lag=1, lag_f=1, ring_slack=6)


CASES = {
    "fp32 f+K, warp-specialised": dict(precision="fp32-mixed", split=True, sweep="fk"),
    "fp32 f+K, mixed kernel": dict(precision="fp32-mixed", split=False, sweep="fk"),
    "fp64 f+K": dict(precision="fp64", split=False, sweep="fk"),
    "fp32 K.v": dict(precision="fp32-mixed", split=False, sweep="kv"),
}


def _run(asm, u, case, check_status=True):
    if case["sweep"] == "kv":
        return asm.kv(u, u, precision=case["precision"], check_status=check_status)
    return asm.assemble(u, precision=case["precision"], check_status=check_status)


@pytest.mark.parametrize("name", list(CASES))
def test_unsatisfiable_wait_gives_up_and_raises(name):
    case = CASES[name]
    m, u = _cube()
    asm = GPUAssembler(m.nodes, m.elements, _material(), precision=case["precision"])
    _small_ring(asm)
    asm.set_queue(split=case["split"])
    key = "btiles_k" if case["sweep"] == "fk" else "btiles_f"
    btiles = asm.dev[key]
    assert asm.dev["plan"].n_granules > 16
    good = btiles.clone()
    btiles[0] = 1 << 30  # no gather can ever publish that many tiles of granule 0
    asm.set_wait_limit(SHORT_WAIT)
    with pytest.raises(RuntimeError, match="bounded wait"):
        _run(asm, u, case)
    torch.cuda.synchronize()  # the launch returned: the context is usable
    assert asm.status_counts()[3] & 1
    # plan restored, default limit: the same bits as a fresh assembler
    btiles.copy_(good)
    asm.set_wait_limit(0)
    got = _run(asm, u, case)
    ref_asm = GPUAssembler(m.nodes, m.elements, _material(), precision=case["precision"])
    _small_ring(ref_asm)
    ref_asm.set_queue(split=case["split"])
    ref = _run(ref_asm, u, case)
    got = got if isinstance(got, tuple) else (got,)
    ref = ref if isinstance(ref, tuple) else (ref,)
    for a, b in zip(got, ref):
        assert torch.equal(a, b)
    assert asm.status_counts()[3] == 0


def test_short_limit_alone_does_not_fail_a_valid_assembly():
    # with the real targets every wait is satisfied eventually: a limit of a few thousand
    # polls still lets a valid assembly complete (waits are short on a quiet queue)
    m, u = _cube(12)
    asm = GPUAssembler(m.nodes, m.elements, _material(), precision="fp32-mixed")
    ref = asm.assemble(u)
    asm.set_wait_limit(1 << 20)
    got = asm.assemble(u)
    assert torch.equal(got[0], ref[0]) and torch.equal(got[1], ref[1])


def test_batched_newton_raises_when_a_wait_gives_up():
    from psierra_b200.batched import BatchedNewton, MeshBatch

    meshes, mus, kappas, forces, fixed = [], [], [], [], []
    for i in range(6):
        m = meshgen.box_tet4(1.0 + 0.1 * i, 0.1, 0.1, 60, 5, 5)  # 9,000 Tet4 each
        mu, _, kappa = meshgen.lame_from_young_poisson(1e5, 0.3)
        clamp = meshgen.nodes_on_plane(m, 0, "min")
        meshes.append(m)
        mus.append(mu)
        kappas.append(kappa)
        forces.append(meshgen.traction_nodal_forces(m, 0, "max", [50.0, 0.0, -10.0]))
        fixed.append(np.concatenate([3 * clamp + c for c in range(3)]))
    batch = MeshBatch(meshes, mus, kappas, precision="fp32-mixed")
    batch.asm.set_queue(lag=1, ring_slack=6)  # ring of 8 granules; the union has 14
    assert batch.asm.dev["plan"].n_granules > 8
    solver = BatchedNewton(batch, fixed, pcg_iterations=20, use_graph=True)
    f_ext = batch.concat(forces)
    batch.asm.dev["btiles_k"][0] = 1 << 30
    batch.asm.set_wait_limit(SHORT_WAIT)
    with pytest.raises(RuntimeError, match="bounded wait"):
        solver.solve(f_ext, n_steps=1, nr_iterations=2)
    torch.cuda.synchronize()


@pytest.mark.parametrize("precision", ["fp64", "fp32-mixed"])
def test_nan_displacement_propagates_like_the_reference(precision):
    m = meshgen.box_tet4(1.0, 0.3, 0.2, 10, 3, 2)
    u = meshgen.cantilever_seeded_u(m, seed=3)
    bad_node = 40
    u[bad_node, 1] = np.nan
    el = Tet4TotalLagrangian(_material(1e5, 0.3), precision=precision)
    f, K = el.assemble_force_and_tangent(m, u)  # no exception, like the reference
    touched = np.unique(m.elements[np.any(m.elements == bad_node, axis=1)])
    want = np.zeros(m.n_nodes, dtype=bool)
    want[touched] = True
    got = ~np.isfinite(f.reshape(-1, 3)).all(axis=1)
    assert np.array_equal(got, want)
    # rows of the touched nodes carry NaN; every other row is finite
    rows_bad = np.repeat(want, 3)
    row_of = np.repeat(np.arange(3 * m.n_nodes), np.diff(K.indptr))
    assert np.isfinite(K.data[~rows_bad[row_of]]).all()
    assert not np.isfinite(K.data[rows_bad[row_of]]).all()
