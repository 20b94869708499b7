"""Batched meshes: one launch for many uneven meshes, Newton as a CUDA graph (GPU)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import rel_2
from psierra_b200 import meshgen
from psierra_b200.assembler import GPUAssembler
from psierra_b200.batched import BatchedNewton, MeshBatch
from psierra_b200.material import NeoHookeanField
from psierra_b200.newton import DeviceNewton

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda")


def small_batch(n=10, seed=11):
    rng = np.random.default_rng(seed)
    cases = []
    for _ in range(n):
        nx = int(rng.integers(3, 14))
        ny = int(rng.integers(1, 4))
        L = float(rng.uniform(0.5, 2.0))
        m = meshgen.box_tet4(L, 0.1, 0.1, nx, ny, ny)
        E = float(rng.uniform(1e3, 1e6))
        nu = float(rng.uniform(0.3, 0.45))
        mu, lam, kappa = meshgen.lame_from_young_poisson(E, nu)
        t = float(rng.uniform(10.0, 1000.0))
        tz = min(0.5 * t, E / (1600.0 * L * L))
        f = meshgen.traction_nodal_forces(m, 0, "max", [t * 0.2, 0.0, -tz])
        clamp = meshgen.nodes_on_plane(m, 0, "min")
        fixed = np.concatenate([3 * clamp + c for c in range(3)])
        cases.append((m, mu, kappa, f, fixed))
    return cases


def single(m, mu, kappa):
    return GPUAssembler(m.nodes, m.elements, NeoHookeanField(np.full(m.n_elements, mu), np.full(m.n_elements, kappa)))


def test_batched_assembly_equals_per_mesh_assembly():
    cases = small_batch()
    mb = MeshBatch([c[0] for c in cases], [c[1] for c in cases], [c[2] for c in cases], precision="fp64")
    rng = np.random.default_rng(0)
    us = [1e-3 * rng.normal(size=c[0].n_dofs) for c in cases]
    fb, kb = mb.asm.assemble(mb.concat(us), precision="fp64")
    fparts = mb.split(fb)
    indptr = mb.asm.pattern.indptr
    for i, (m, mu, kappa, _, _) in enumerate(cases):
        a = single(m, mu, kappa)
        f1, k1 = a.assemble(torch.from_numpy(us[i]).to(DEV), precision="fp64")
        assert torch.equal(fparts[i], f1)
        # the union's CSR is block diagonal: instance i's rows hold exactly its own pattern
        o = int(mb.dof_offsets[i])
        lo, hi = int(indptr[o]), int(indptr[o + 3 * m.n_nodes])
        assert hi - lo == a.nnz
        assert torch.equal(kb[lo:hi], k1)


@pytest.mark.parametrize("precision", ["fp64", "fp32-mixed"])
def test_batched_newton_matches_per_instance_newton(precision):
    cases = small_batch()
    mb = MeshBatch([c[0] for c in cases], [c[1] for c in cases], [c[2] for c in cases], precision=precision)
    bn = BatchedNewton(mb, [c[4] for c in cases], pcg_iterations=3000, pcg_rtol=1e-10)
    res = bn.solve(mb.concat([c[3] for c in cases]), n_steps=4, nr_iterations=30, nr_tol=1e-8)
    assert res.converged.all()
    assert (res.iterations > 0).all()
    for i, (m, mu, kappa, f, fixed) in enumerate(cases):
        dn = DeviceNewton(single(m, mu, kappa), fixed, precision="fp64", pcg_tol=1e-12)
        r1 = dn.solve(torch.from_numpy(f).to(DEV), n_steps=4, nr_iterations=30, nr_tol=1e-10)
        assert r1.converged
        assert rel_2(res.u[i].cpu().numpy(), r1.u.cpu().numpy()) < 1e-6, i


def test_graph_replay_is_bitwise_equal_to_eager_iteration():
    cases = small_batch(n=6, seed=3)
    mb = MeshBatch([c[0] for c in cases], [c[1] for c in cases], [c[2] for c in cases], precision="fp32-mixed")
    f = mb.concat([c[3] for c in cases])
    out = []
    for use_graph in (True, False):
        bn = BatchedNewton(mb, [c[4] for c in cases], pcg_iterations=800, use_graph=use_graph)
        res = bn.solve(f, n_steps=2, nr_iterations=12, nr_tol=1e-8)
        out.append((torch.cat(res.u), res.iterations.copy(), res.replays))
    assert torch.equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1]) and out[0][2] == out[1][2]


def test_autotuner_keeps_results_bitwise_and_caches(tmp_path):
    from psierra_b200 import autotune

    m = meshgen.box_tet4(1.0, 1.0, 1.0, 14, 14, 14)
    u = torch.from_numpy(meshgen.cube_smooth_u(m, seed=1).reshape(-1)).to(DEV)
    mu, lam, kappa = meshgen.lame_from_young_poisson(3e3, 0.45)
    a = GPUAssembler(m.nodes, m.elements, NeoHookeanField(np.full(m.n_elements, mu), np.full(m.n_elements, kappa)),
                     precision="fp32-mixed")
    f0, k0 = a.assemble(u)
    f0, k0 = f0.clone(), k0.clone()
    cache = str(tmp_path / "tune.json")
    best = autotune.tune(a, u, lags=(2, 8), blocks=(1, 2), slacks=(6, 16), reps=2, cache_file=cache)
    # every schedule, mixed or warp-specialised, gives the same bits
    assert len(best["table"]) == 16 and best["ms"] > 0
    f1, k1 = a.assemble(u)
    assert torch.equal(f0, f1) and torch.equal(k0, k1)
    for lag, bps, slack, split in best["table"]:
        a.set_queue(lag=lag, blocks_per_sm=bps, ring_slack=slack, split=split)
        f2, k2 = a.assemble(u)
        assert torch.equal(f0, f2) and torch.equal(k0, k2)
        _, k3 = a.assemble(u, want_f=False)
        assert torch.equal(k0, k3)
    # the f / K.v queue has its own lag
    y0 = a.kv(u, u).clone()
    for lag_f in (4, 24):
        a.set_queue(lag_f=lag_f)
        assert torch.equal(a.kv(u, u), y0)
    autotune._cache.clear()
    again = autotune.tune(a, u, cache_file=cache)
    assert again["ms"] is None
    assert (again["lag"], again["blocks_per_sm"], again["ring_slack"], again["split"]) == (
        best["lag"], best["blocks_per_sm"], best["ring_slack"], best["split"])
