"""The row-sampling oracle against the complete oracle assembly (CPU).

``oracle.sample.sampled_rows`` evaluates only the elements incident to the sampled nodes;
their rows must equal the complete assembly's bit for bit (same elements, same element
order in the COO->CSR summation).
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle import sample as osample
from oracle import vectorized
from psierra_b200 import meshgen


@pytest.mark.parametrize("tet10", [False, True], ids=["Tet4", "Tet10"])
def test_sampled_rows_equal_complete_assembly(tet10):
    m = meshgen.box_tet4(1.0, 0.6, 0.4, 6, 4, 3)
    if tet10:
        m = meshgen.tet4_to_tet10(m)
    u = meshgen.cube_smooth_u(m, seed=3)
    mu = np.random.default_rng(1).uniform(1e3, 2e3, m.n_elements)
    f_all, K_all = vectorized.assemble_force_and_tangent(m.nodes, m.elements, u, mu, 20.0 * mu)
    nodes = osample.sample_nodes(m.n_nodes, 25, seed=9)
    dofs, K, f = osample.sampled_rows(m.nodes, m.elements, u, mu, 20.0 * mu, nodes, chunk=50)
    assert np.array_equal(dofs, np.sort(np.concatenate([3 * nodes + c for c in range(3)])))
    ref = K_all[dofs]
    ref.sort_indices()
    K.sort_indices()
    assert np.array_equal(K.indptr, ref.indptr) and np.array_equal(K.indices, ref.indices)
    assert np.array_equal(K.data, ref.data)
    assert np.array_equal(f, f_all[dofs])
    same, err = osample.compare_rows(osample.gpu_rows(K_all.indptr, K_all.indices, K_all.data, dofs), K)
    assert same and err == 0.0
