"""The allocation-free CG entry point (psx_pcg_static) against the workspace one (psx_pcg).

psx_pcg_static serves callers that cannot allocate device memory when they solve: its
scratch is a fixed array inside the library.  This file is named so that pytest
collects it last; it also passes on its own in a fresh process.  Both entry points are
called through the C ABI (ctypes), on the reference's cfg1 tangent restricted to its
free DOFs, twice in a row for the static one (the second call runs on scratch the
first one left behind).
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest
import scipy.sparse as spsp
import torch

from conftest import golden, rel_2
from psierra_b200 import _lib, meshgen

pytestmark = pytest.mark.gpu

_p, _i64, _i32, _f64 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_double


def _bind():
    L = _lib.lib()
    L.psx_pcg_static.argtypes = [_i64, _p, _p, _p, _i32, _p, _p, _f64, _f64, _i32, _i32, _p, _p]
    L.psx_pcg_static.restype = ctypes.c_int
    L.psx_pcg_static_max_bytes.argtypes = []
    L.psx_pcg_static_max_bytes.restype = ctypes.c_size_t
    return L


def _system(node_aligned: bool):
    g = golden("cfg1_seeded")
    m = meshgen.box_tet4(1.0, 0.1, 0.1, 40, 4, 4)
    K = spsp.csr_matrix((g["K_data"], g["K_indices"], g["K_indptr"]), shape=(m.n_dofs, m.n_dofs))
    clamp = meshgen.nodes_on_plane(m, 0, "min")
    fixed = np.sort(np.concatenate([3 * clamp + c for c in range(3)]))
    f = meshgen.traction_nodal_forces(m, 0, "max", [0.0, 0.0, -500.0])
    if not node_aligned:
        free = np.setdiff1d(np.arange(m.n_dofs), fixed)
        return K[free, :][:, free].tocsr(), f[free]
    mask = np.ones(m.n_dofs)
    mask[fixed] = 0.0
    D = spsp.diags(mask)
    A = (D @ K @ D + spsp.diags(1.0 - mask)).tocsr()
    A.sort_indices()
    b = f.copy()
    b[fixed] = 0.0
    return A, b


def _device(A, b):
    d = torch.device("cuda")
    return (torch.from_numpy(A.indptr.astype(np.int32)).to(d), torch.from_numpy(A.indices.astype(np.int32)).to(d),
            torch.from_numpy(A.data.astype(np.float64)).to(d), torch.from_numpy(b).to(d))


def _solve_workspace(L, n, dev, precond):
    indptr, indices, vals, b = dev
    nbytes = ctypes.c_int64()
    assert L.psx_pcg_work_bytes(n, precond, ctypes.byref(nbytes)) == _lib.PSX_OK
    work = torch.empty(int(nbytes.value), dtype=torch.uint8, device="cuda")
    st = torch.zeros(8, dtype=torch.int32, device="cuda")
    x = torch.zeros_like(b)
    rc = L.psx_pcg(n, indptr.data_ptr(), indices.data_ptr(), vals.data_ptr(), _lib.PSX_FP64, b.data_ptr(),
                   x.data_ptr(), 1e-10, 0.0, 20000, precond, work.data_ptr(), work.numel(), st.data_ptr(),
                   torch.cuda.current_stream().cuda_stream)
    assert rc == _lib.PSX_OK
    return x.cpu().numpy(), st.cpu()


def _solve_static(L, n, dev, precond):
    indptr, indices, vals, b = dev
    st = torch.zeros(8, dtype=torch.int32, device="cuda")
    x = torch.zeros_like(b)
    rc = L.psx_pcg_static(n, indptr.data_ptr(), indices.data_ptr(), vals.data_ptr(), _lib.PSX_FP64,
                          b.data_ptr(), x.data_ptr(), 1e-10, 0.0, 20000, precond, st.data_ptr(),
                          torch.cuda.current_stream().cuda_stream)
    assert rc == _lib.PSX_OK
    return x.cpu().numpy(), st.cpu()


@pytest.mark.parametrize("precond,aligned", [(_lib.PSX_PRECOND_JACOBI, False), (_lib.PSX_PRECOND_BJACOBI, True)])
def test_static_scratch_matches_workspace_entry_point(precond, aligned):
    L = _bind()
    A, b = _system(aligned)
    n = A.shape[0]
    dev = _device(A, b)
    x_ref, st_ref = _solve_workspace(L, n, dev, precond)
    assert int(st_ref[5]) == 0  # converged
    for _ in range(2):  # two calls in a row share the scratch array
        x, st = _solve_static(L, n, dev, precond)
        assert int(st[5]) == 0 and int(st[4]) == int(st_ref[4])
        assert rel_2(x, x_ref) < 1e-12
    assert np.linalg.norm(A @ x - b) < 1e-9 * np.linalg.norm(b)


def test_static_call_after_the_first_reserves_no_device_memory():
    # the first call has loaded the module and looked up the scratch address; a later
    # call must leave the device's free memory unchanged (its outputs are allocated first)
    L = _bind()
    A, b = _system(False)
    n = A.shape[0]
    indptr, indices, vals, bd = _device(A, b)
    st = torch.zeros(8, dtype=torch.int32, device="cuda")
    x = torch.zeros_like(bd)
    stream = torch.cuda.current_stream().cuda_stream

    def call():
        rc = L.psx_pcg_static(n, indptr.data_ptr(), indices.data_ptr(), vals.data_ptr(), _lib.PSX_FP64,
                              bd.data_ptr(), x.data_ptr(), 1e-10, 0.0, 20000, _lib.PSX_PRECOND_JACOBI,
                              st.data_ptr(), stream)
        assert rc == _lib.PSX_OK
        torch.cuda.synchronize()

    call()
    free_before, _ = torch.cuda.mem_get_info()
    call()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before
    assert int(st[5].item()) == 0


def test_static_scratch_rejects_systems_beyond_its_size():
    L = _bind()
    cap = int(L.psx_pcg_static_max_bytes())
    assert cap == 32 << 20
    A, b = _system(False)
    dev = _device(A, b)
    indptr, indices, vals, bd = dev
    st = torch.zeros(8, dtype=torch.int32, device="cuda")
    x = torch.zeros_like(bd)
    too_big = 1_000_000  # needs ~40 MB of scratch with Jacobi
    need = ctypes.c_int64()
    assert L.psx_pcg_work_bytes(too_big, _lib.PSX_PRECOND_JACOBI, ctypes.byref(need)) == _lib.PSX_OK
    assert need.value > cap
    rc = L.psx_pcg_static(too_big, indptr.data_ptr(), indices.data_ptr(), vals.data_ptr(), _lib.PSX_FP64,
                          bd.data_ptr(), x.data_ptr(), 1e-10, 0.0, 10, _lib.PSX_PRECOND_JACOBI, st.data_ptr(),
                          torch.cuda.current_stream().cuda_stream)
    assert rc == _lib.PSX_ERR_LIMIT
