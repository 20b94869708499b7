"""The throughput form of the drop-in element (CPU, with a fake assembler in place of the
GPU one): f and K_T stay tensors, K_T as a ``DeviceCSR`` over the pattern's arrays, and
``to_scipy`` gives the canonical float64 CSR of the parity-mode hooks."""
from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse as spsp
import torch

from psierra_b200.element import DeviceCSR, Tet4Fbar, Tet4TotalLagrangian


class FakeAssembler:
    def __init__(self, A: spsp.csr_matrix, f: np.ndarray, dtype=torch.float32):
        self.n_nodes = A.shape[0] // 3
        self.dev = {"indptr": torch.from_numpy(A.indptr.astype(np.int32)),
                    "indices": torch.from_numpy(A.indices.astype(np.int32))}
        self._vals, self._f = torch.from_numpy(A.data).to(dtype), torch.from_numpy(f)
        self.seen = []

    def assemble(self, u, want_f=True, want_k=True):
        self.seen.append(u)
        return self._f.clone(), self._vals.clone()


def _problem():
    rng = np.random.default_rng(3)
    A = spsp.random(12, 12, density=0.4, random_state=4, format="csr") + spsp.identity(12, format="csr")
    A = (A + A.T).tocsr()
    A.sort_indices()
    return A, rng.standard_normal(12)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_device_form_keeps_tensors_and_converts_to_the_canonical_csr(monkeypatch, dtype):
    A, f_ref = _problem()
    fake = FakeAssembler(A, f_ref, dtype)
    el = Tet4TotalLagrangian(material=None)
    monkeypatch.setattr(el, "_setup", lambda mesh: fake)
    u = torch.arange(12, dtype=torch.float64).reshape(4, 3)
    f, K = el.assemble_force_and_tangent_device(object(), u)
    assert isinstance(f, torch.Tensor) and isinstance(K, DeviceCSR)
    assert fake.seen[0].shape == (12,) and fake.seen[0].data_ptr() == u.data_ptr()  # no copy of a device u
    assert K.shape == (12, 12) and K.nnz == A.nnz and K.data.dtype == dtype
    assert K.indptr is fake.dev["indptr"] and K.indices is fake.dev["indices"]
    B = K.to_scipy()
    assert B.data.dtype == np.float64 and B.has_canonical_format
    assert np.array_equal(B.indptr, A.indptr) and np.array_equal(B.indices, A.indices)
    np.testing.assert_array_equal(B.data, A.data.astype(np.float32 if dtype == torch.float32 else np.float64))
    np.testing.assert_array_equal(f.numpy(), f_ref)


def test_host_displacement_is_uploaded(monkeypatch):
    A, f_ref = _problem()
    fake = FakeAssembler(A, f_ref)
    el = Tet4TotalLagrangian(material=None)
    monkeypatch.setattr(el, "_setup", lambda mesh: fake)
    uploaded = []
    monkeypatch.setattr(el, "_upload_u", lambda d: uploaded.append(d) or torch.zeros(12, dtype=torch.float64))
    u_host = np.ones((4, 3))
    el.assemble_force_and_tangent_device(object(), u_host)
    assert uploaded and uploaded[0] is u_host


def test_fbar_has_no_device_form():
    with pytest.raises(NotImplementedError, match="host only"):
        Tet4Fbar(material=None).assemble_force_and_tangent_device(object(), np.zeros((4, 3)))
