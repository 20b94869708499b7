"""GPU parity against the oracle at the benchmarked sizes (many granules, wrapped rings).

The smaller assembly tests fit in one 4,096-element granule, where the persistent
queue never waits across granules and the ring of element / tile records never wraps.
Here the meshes span tens of granules:

* the 40^3 cube (384,000 Tet4, 94 granules) against the complete oracle assembly
  (psierra ``element/tet4_total_lagrangian.py:77-139`` + ``utility/assembly.py:37-108``),
  with the default queue and with a ring shrunk to 16 granules so that it wraps 5 times, for the FP64 kernel and for both FP32-tangent kernels;
* a 14^3 Tet10 cube (16,464 elements, 33 granules of 512) against the complete oracle;
* the headline workload itself (80^3 cube, 3,072,000 Tet4) and the 162,000-Tet10 cube
  on a seeded sample of rows (``oracle.sample``: the elements incident to the sampled
  nodes give those rows exactly).

Tolerances: FP64 K_T max-relative and f_int 2-norm relative <= 1e-12 (the plain mode's
bar); FP32-mixed K_T <= 1e-6 (f_int stays FP64: <= 1e-12).  CSR index arrays are
compared byte for byte.
"""
from __future__ import annotations

import functools

import numpy as np
import pytest
import torch

from conftest import rel_2, rel_max
from oracle import sample as osample
from oracle import vectorized
from oracle.assembly import assemble_sparse, assemble_vector, coo_indices, element_dofs
from psierra_b200 import meshgen
from psierra_b200.assembler import GPUAssembler
from psierra_b200.material import IsotropicElasticParameters, NeoHookean

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda")
FP64_TOL = 1e-12
MIXED_TOL = 1e-6


def _material(E, nu):
    p = IsotropicElasticParameters()
    p.set_from_youngs_poisson(youngs_modulus=E, poissons_ratio=nu, mass_density=1000.0)
    return NeoHookean(p)


@functools.lru_cache(maxsize=None)
def _tet4_cube(cells):
    m = meshgen.box_tet4(1.0, 1.0, 1.0, cells, cells, cells)
    return m, meshgen.cube_smooth_u(m, seed=2024), _material(3e3, 0.45)


@functools.lru_cache(maxsize=None)
def _tet10_cube(cells):
    m = meshgen.tet4_to_tet10(meshgen.box_tet4(1.0, 1.0, 1.0, cells, cells, cells))
    return m, meshgen.cube_smooth_u(m, seed=7), _material(1e4, 0.4)


@functools.lru_cache(maxsize=None)
def _oracle_full(kind, cells):
    m, u, mat = (_tet4_cube if kind == "tet4" else _tet10_cube)(cells)
    mu, kappa = mat.parameters.shear_modulus, mat.parameters.bulk_modulus
    ks, fs = [], []
    for a in range(0, m.n_elements, 50000):
        k, f = vectorized.element_force_and_tangent(m.nodes, m.elements[a:a + 50000], u, mu, kappa)
        ks.append(k)
        fs.append(f)
    ed = element_dofs(m.elements)
    r, c = coo_indices(ed)
    K = assemble_sparse(np.concatenate(ks), r, c, m.n_dofs)
    f = assemble_vector(np.concatenate(fs), ed, m.n_dofs)
    return K, f


def _gpu(m, u, mat, precision, split=None, small_ring=False):
    a = GPUAssembler(m.nodes, m.elements, mat, precision=precision)
    if small_ring:
        a.set_queue(lag=2, lag_f=2, ring_slack=6)
    if split is not None:
        a.set_queue(split=split)
    f, k = a.assemble(torch.from_numpy(u.reshape(-1)).to(DEV))
    assert a.status_counts() == (0, 0, -1, 0)
    return a, f.cpu().numpy(), k.double().cpu().numpy()


TET4_CASES = {
    "fp64": ("fp64", None),
    "fp32 warp-specialised": ("fp32-mixed", True),
    "fp32 mixed kernel": ("fp32-mixed", False),
}


@pytest.mark.parametrize("small_ring", [False, True], ids=["default ring", "small ring"])
@pytest.mark.parametrize("name", list(TET4_CASES))
def test_tet4_cube40_matches_oracle(name, small_ring):
    precision, split = TET4_CASES[name]
    m, u, mat = _tet4_cube(40)
    K_ref, f_ref = _oracle_full("tet4", 40)
    a, f, k = _gpu(m, u, mat, precision, split, small_ring)
    if small_ring:
        assert a.dev["plan"].n_granules == 94  # over a ring of 16 granules: it wraps 5 times
    assert np.array_equal(a.pattern.indptr, K_ref.indptr) and np.array_equal(a.pattern.indices, K_ref.indices)
    tol = FP64_TOL if precision == "fp64" else MIXED_TOL
    assert rel_max(k, K_ref.data) < tol
    assert rel_2(f, f_ref) < FP64_TOL


@pytest.mark.parametrize("small_ring", [False, True], ids=["default ring", "small ring"])
@pytest.mark.parametrize("precision", ["fp64", "fp32-mixed"])
def test_tet10_cube14_matches_oracle(precision, small_ring):
    m, u, mat = _tet10_cube(14)
    K_ref, f_ref = _oracle_full("tet10", 14)
    a, f, k = _gpu(m, u, mat, precision, None, small_ring)
    assert a.dev["plan"].n_granules == 33
    assert np.array_equal(a.pattern.indptr, K_ref.indptr) and np.array_equal(a.pattern.indices, K_ref.indices)
    tol = FP64_TOL if precision == "fp64" else MIXED_TOL
    assert rel_max(k, K_ref.data) < tol
    assert rel_2(f, f_ref) < FP64_TOL


@functools.lru_cache(maxsize=None)
def _oracle_rows(kind, cells, count, seed):
    m, u, mat = (_tet4_cube if kind == "tet4" else _tet10_cube)(cells)
    nodes = osample.sample_nodes(m.n_nodes, count, seed)
    return osample.sampled_rows(m.nodes, m.elements, u, mat.parameters.shear_modulus,
                                mat.parameters.bulk_modulus, nodes)


@pytest.mark.parametrize("precision", ["fp64", "fp32-mixed"])
@pytest.mark.parametrize("kind,cells", [("tet4", 80), ("tet10", 30)], ids=["cube80 Tet4", "cube30 Tet10"])
def test_full_size_sampled_rows_match_oracle(kind, cells, precision):
    m, u, mat = (_tet4_cube if kind == "tet4" else _tet10_cube)(cells)
    dofs, K_ref, f_ref = _oracle_rows(kind, cells, 1500, 17)
    a, f, k = _gpu(m, u, mat, precision)
    same, err = osample.compare_rows(osample.gpu_rows(a.pattern.indptr, a.pattern.indices, k, dofs), K_ref)
    assert same
    assert err < (FP64_TOL if precision == "fp64" else MIXED_TOL)
    assert rel_2(f[dofs], f_ref) < FP64_TOL
