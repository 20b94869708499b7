"""Warp-specialised Tet4 FP32 tangent kernel (GPU).

Element tiles and gathers run in separate warps of one block per SM; each K and f entry
is still summed by one owner in the fixed contribution order, so the kernel must give
the same bits as the mixed kernel (whose parity with the oracle the assembly tests pin)
on any mesh: ragged element counts, disjoint unions of uneven meshes, a cube large
enough that the ring of tile records wraps many times.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from psierra_b200 import _lib, meshgen
from psierra_b200.assembler import GPUAssembler
from psierra_b200.material import NeoHookeanField

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda")


def _beams():
    union, _, _ = meshgen.concat_meshes([c.mesh for c in meshgen.beam_batch(n=12, target_tets=60000, seed=3)])
    return union


MESHES = {
    "ragged box": lambda: meshgen.box_tet4(1.0, 0.3, 0.5, 7, 3, 5),
    "12 uneven beams": _beams,
    "cube 40": lambda: meshgen.box_tet4(1.0, 1.0, 1.0, 40, 40, 40),
}


def test_split_kernel_is_available():
    assert _lib.lib().psx_tet4_split_ready() == 1


@pytest.mark.parametrize("name", list(MESHES))
def test_split_kernel_equals_mixed_kernel_bitwise(name):
    mesh = MESHES[name]()
    rng = np.random.default_rng(4)
    E = mesh.n_elements
    mu = rng.uniform(1e3, 5e3, E)
    a = GPUAssembler(mesh.nodes, mesh.elements, NeoHookeanField(mu, 20.0 * mu), precision="fp32-mixed")
    X = mesh.nodes
    ext = float(np.ptp(X, axis=0).max())
    # smooth field (3 % shear plus a small wave): no element inverts
    uf = 0.03 * (X[:, [1, 2, 0]] - X.mean(axis=0)) + 0.002 * ext * np.sin(6.0 * X / ext)
    u = torch.from_numpy(np.ascontiguousarray(uf).reshape(-1)).to(DEV)
    out = {}
    for split in (False, True):
        a.set_queue(split=split)
        f, k = a.assemble(u)
        _, kk = a.assemble(u, want_f=False)
        assert int(a.status[0].item()) == 0  # no bounded wait gave up
        out[split] = (f.clone(), k.clone(), kk.clone())
    for x, y in zip(out[False], out[True]):
        assert torch.equal(x, y), name
    # repeated calls reuse the counters and the ring: still the same bits
    f2, k2 = a.assemble(u)
    assert torch.equal(f2, out[True][0]) and torch.equal(k2, out[True][1])


@pytest.mark.parametrize("name", ["ragged box", "cube 40"])
def test_effective_tangent_split_equals_mixed_kernel_bitwise(name):
    """c_t K_T + c_m M + c_0 K_0 (the dynamic effective tangent) through the
    warp-specialised kernel gives the mixed kernel's bits."""
    mesh = MESHES[name]()
    E = mesh.n_elements
    mu = np.random.default_rng(5).uniform(1e3, 5e3, E)
    a = GPUAssembler(mesh.nodes, mesh.elements, NeoHookeanField(mu, 20.0 * mu, mass_density=1000.0),
                     precision="fp32-mixed")
    X = mesh.nodes
    uf = 0.02 * (X[:, [2, 0, 1]] - X.mean(axis=0))
    u = torch.from_numpy(np.ascontiguousarray(uf).reshape(-1)).to(DEV)
    out = {}
    for split in (False, True):
        a.set_queue(split=split)
        f, k = a.assemble_effective(u, 0.9, 37.0, 0.0)
        _, kk = a.assemble_effective(u, 0.9, 37.0, 0.0, want_f=False)
        out[split] = (f.clone(), k.clone(), kk.clone())
    for x, y in zip(out[False], out[True]):
        assert torch.equal(x, y), name
