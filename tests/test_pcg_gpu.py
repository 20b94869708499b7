"""GPU PCG against scipy's cg (the reference ConjugateGradientSolver) and SuperLU.

System: the reference's assembled K_T at the cfg1 seeded state (golden values),
restricted to the free DOFs exactly as NonlinearStaticAnalysis slices it
(psierra analysis/nonlinear_static.py:354-355).
"""
from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse as spsp
import scipy.sparse.linalg as spla
import torch

from conftest import golden, rel_2
from psierra_b200 import meshgen
from psierra_b200.solver import ConjugateGradientSolver

pytestmark = pytest.mark.gpu


def free_system():
    g = golden("cfg1_seeded")
    m = meshgen.box_tet4(1.0, 0.1, 0.1, 40, 4, 4)
    K = spsp.csr_matrix((g["K_data"], g["K_indices"], g["K_indptr"]), shape=(m.n_dofs, m.n_dofs))
    clamp = meshgen.nodes_on_plane(m, 0, "min")
    fixed = np.sort(np.concatenate([3 * clamp + c for c in range(3)]))
    free = np.setdiff1d(np.arange(m.n_dofs), fixed)
    Kf = K[free, :][:, free].tocsr()
    b = meshgen.traction_nodal_forces(m, 0, "max", [0.0, 0.0, -500.0])[free]
    return K, Kf, b, free


def scipy_cg(A, b, rtol, maxiter):
    diag = A.diagonal()
    inv = np.where(np.abs(diag) > 1e-14, 1.0 / diag, 1.0)
    M = spla.LinearOperator(A.shape, matvec=lambda x: inv * x)
    its = [0]
    x, info = spla.cg(A, b, M=M, rtol=rtol, maxiter=maxiter, callback=lambda xk: its.__setitem__(0, its[0] + 1))
    return x, info, its[0]


def test_jacobi_pcg_matches_scipy_cg_and_superlu():
    _, Kf, b, _ = free_system()
    x_ref, info, its = scipy_cg(Kf, b, 1e-10, 20000)
    assert info == 0
    solver = ConjugateGradientSolver(tolerance=1e-10, max_iterations=20000)
    x = solver.solve(Kf, b)
    assert solver.last.converged
    # same recurrence; on this ill-conditioned cantilever, rounding of the dot products
    # (fixed-tree on the GPU, pairwise in numpy) moves the iteration count by a few percent
    assert abs(solver.last.iterations - its) <= max(3, its // 20)
    # the true residual drifts from the recursive one over ~900 iterations, for scipy too
    assert np.linalg.norm(Kf @ x - b) < max(1e-9 * np.linalg.norm(b), 10 * np.linalg.norm(Kf @ x_ref - b))
    assert rel_2(x, x_ref) < 1e-7
    x_lu = spla.spsolve(Kf.tocsc(), b)
    assert rel_2(x, x_lu) < 1e-6


def test_pcg_is_bitwise_reproducible_and_reports_nonconvergence():
    _, Kf, b, _ = free_system()
    s = ConjugateGradientSolver(tolerance=1e-9, max_iterations=5000)
    x1 = s.solve(Kf, b)
    x2 = s.solve(Kf, b)
    assert np.array_equal(x1, x2)
    with pytest.raises(RuntimeError, match="Conjugate Gradient did not converge"):
        ConjugateGradientSolver(tolerance=1e-12, max_iterations=5).solve(Kf, b)


def test_block_jacobi_on_node_aligned_system():
    K, _, b_free, free = free_system()
    n = K.shape[0]
    fixed = np.setdiff1d(np.arange(n), free)
    # symmetric elimination of the clamped DOFs keeps the node-aligned layout
    mask = np.ones(n)
    mask[fixed] = 0.0
    D = spsp.diags(mask)
    A = (D @ K @ D + spsp.diags(1.0 - mask)).tocsr()
    A.sort_indices()
    b = np.zeros(n)
    b[free] = b_free
    sj = ConjugateGradientSolver(tolerance=1e-10, max_iterations=20000, preconditioner="jacobi")
    sb = ConjugateGradientSolver(tolerance=1e-10, max_iterations=20000, preconditioner="block-jacobi")
    xj = sj.solve(A, b)
    xb = sb.solve(A, b)
    assert sb.last.converged and sb.last.iterations <= sj.last.iterations
    x_lu = spla.spsolve(A.tocsc(), b)
    assert rel_2(xb, x_lu) < 1e-6 and rel_2(xj, x_lu) < 1e-6


def test_fp32_matrix_values():
    _, Kf, b, _ = free_system()
    dev = torch.device("cuda")
    s = ConjugateGradientSolver(tolerance=1e-8, max_iterations=20000)
    x = torch.zeros(len(b), dtype=torch.float64, device=dev)
    res = s.solve_device(torch.from_numpy(Kf.indptr.astype(np.int32)).to(dev),
                         torch.from_numpy(Kf.indices.astype(np.int32)).to(dev),
                         torch.from_numpy(Kf.data.astype(np.float32)).to(dev),
                         torch.from_numpy(b).to(dev), x)
    assert res.converged
    # the FP32 values define a (slightly) different matrix: compare with its exact solve
    K32 = spsp.csr_matrix((Kf.data.astype(np.float32).astype(np.float64), Kf.indices, Kf.indptr), shape=Kf.shape)
    x_lu = spla.spsolve(K32.tocsc(), b)
    assert rel_2(x.cpu().numpy(), x_lu) < 1e-6


@pytest.mark.parametrize("precond", ["jacobi", "block-jacobi"])
def test_nodal_spmv_matches_row_spmv(precond):
    """PSX_PCG_NODAL (node-blocked SpMV) on the assembler's layout: the same solution as
    the row-wise SpMV (summation order differs, so within rounding) and as SuperLU."""
    from psierra_b200.solver import is_nodal_csr

    K, _, b_free, free = free_system()
    n = K.shape[0]
    fixed = np.setdiff1d(np.arange(n), free)
    # eliminate the clamped DOFs in place, keeping every stored entry (the layout stays)
    A = K.copy().tocsr()
    A.sort_indices()
    rows = np.repeat(np.arange(n), np.diff(A.indptr))
    isfix = np.zeros(n, dtype=bool)
    isfix[fixed] = True
    A.data[isfix[rows] | isfix[A.indices]] = 0.0
    A.data[isfix[rows] & (rows == A.indices)] = 1.0
    assert is_nodal_csr(A.indptr, A.indices)
    b = np.zeros(n)
    b[free] = b_free
    dev = torch.device("cuda")
    t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a, dtype=dt)).to(dev)  # noqa: E731
    xs = {}
    for nodal in (False, True):
        s = ConjugateGradientSolver(tolerance=1e-10, max_iterations=20000, preconditioner=precond)
        x = torch.zeros(n, dtype=torch.float64, device=dev)
        res = s.solve_device(t(A.indptr, np.int32), t(A.indices, np.int32), t(A.data, np.float64), t(b, np.float64), x,
                             nodal=nodal)
        assert res.converged
        xs[nodal] = (x.cpu().numpy(), res.iterations)
    # rounding differs with the summation order: on this ill-conditioned beam the
    # iteration counts move by a few percent, the solutions agree to the solver tolerance
    assert abs(xs[True][1] - xs[False][1]) <= max(2, 0.05 * xs[False][1])
    assert rel_2(xs[True][0], xs[False][0]) < 1e-6
    x_lu = spla.spsolve(A.tocsc(), b)
    assert rel_2(xs[True][0], x_lu) < 1e-6
    # the host entry point detects the layout itself
    s = ConjugateGradientSolver(tolerance=1e-10, max_iterations=20000, preconditioner=precond)
    assert rel_2(s.solve(A, b), x_lu) < 1e-6
