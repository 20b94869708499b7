"""Pooled pinned result arrays of the drop-in element (GPU)."""
from __future__ import annotations

import gc

import numpy as np
import pytest
import torch

from psierra_b200 import meshgen
from psierra_b200.element import Tet4TotalLagrangian
from psierra_b200.material import IsotropicElasticParameters, NeoHookean

pytestmark = pytest.mark.gpu


def test_returned_matrices_are_fresh_and_buffers_are_recycled():
    p = IsotropicElasticParameters()
    p.set_from_youngs_poisson(youngs_modulus=1e4, poissons_ratio=0.3, mass_density=1000.0)
    m = meshgen.box_tet4(1.0, 0.5, 0.5, 6, 3, 3)
    el = Tet4TotalLagrangian(NeoHookean(p), precision="fp32-mixed")
    u1 = meshgen.cantilever_seeded_u(m, seed=1)
    u2 = meshgen.cantilever_seeded_u(m, seed=2)
    K1 = el.assemble_tangent_stiffness_matrix(m, u1)
    K1_copy = K1.data.copy()
    K2 = el.assemble_tangent_stiffness_matrix(m, u2)  # K1 is alive: must not be overwritten
    assert np.array_equal(K1.data, K1_copy)
    assert not np.shares_memory(K1.data, K2.data)
    assert K1.data.dtype == np.float64 and not np.array_equal(K1.data, K2.data)
    # the reference's values: the same as the FP32 values widened
    _, k32 = el._asm.assemble(torch.from_numpy(u2.reshape(-1)).cuda(), want_f=False)
    assert np.array_equal(K2.data, k32.double().cpu().numpy())
    in_use = el._results.in_use_bytes
    del K1
    gc.collect()
    assert el._results.in_use_bytes < in_use  # the buffer went back to the pool
    K3 = el.assemble_tangent_stiffness_matrix(m, u1)
    assert np.array_equal(K3.data, K1_copy)
