"""The pinned result pool behind the drop-in element's returned arrays (CPU; pinned
allocation and the stream are replaced by plain host tensors and a no-op stream).

The reference returns a new array from every assembly; the pool must keep that: two
live results never share memory, a buffer goes back to the pool only when the caller
drops the array that views it, and past the byte cap results are plain fresh arrays."""
from __future__ import annotations

import gc

import numpy as np
import pytest
import torch

from psierra_b200.element import _ResultPool


@pytest.fixture
def host_only(monkeypatch):
    real_empty = torch.empty
    allocs = []

    def empty(*args, pin_memory=False, **kw):
        t = real_empty(*args, **kw)
        if pin_memory:
            allocs.append(t)
        return t

    class _Stream:
        def synchronize(self):
            pass

    monkeypatch.setattr(torch, "empty", empty)
    monkeypatch.setattr(torch.cuda, "current_stream", lambda *a, **k: _Stream())
    return allocs


def test_results_are_fresh_and_buffers_return_on_drop(host_only):
    pool = _ResultPool(cap_bytes=1 << 20)
    a_dev = torch.arange(1000, dtype=torch.float64)
    a = pool.take(a_dev)
    b = pool.take(a_dev * 2)
    np.testing.assert_array_equal(a, np.arange(1000.0))
    np.testing.assert_array_equal(b, 2 * np.arange(1000.0))
    assert not np.shares_memory(a, b)
    assert len(host_only) == 2 and pool.in_use_bytes == 2 * 8000
    del a
    gc.collect()
    assert pool.in_use_bytes == 8000 and len(pool.free) == 1
    c = pool.take(a_dev * 3)  # reuses the dropped buffer: no new allocation
    assert len(host_only) == 2
    np.testing.assert_array_equal(c, 3 * np.arange(1000.0))
    np.testing.assert_array_equal(b, 2 * np.arange(1000.0))  # the live result is untouched
    assert not np.shares_memory(b, c)


def test_buffers_are_matched_by_size(host_only):
    pool = _ResultPool(cap_bytes=1 << 20)
    small = pool.take(torch.ones(10, dtype=torch.float64))
    del small
    gc.collect()
    big = pool.take(torch.ones(20, dtype=torch.float64))
    assert len(host_only) == 2  # the 10-value buffer does not serve a 20-value result
    assert big.shape == (20,) and len(pool.free) == 1


def test_past_the_cap_results_are_plain_arrays(host_only):
    pool = _ResultPool(cap_bytes=8 * 100)
    a = pool.take(torch.full((100,), 1.5, dtype=torch.float64))
    b = pool.take(torch.full((100,), 2.5, dtype=torch.float64))  # over the cap: not pooled
    assert len(host_only) == 1 and pool.in_use_bytes == 800
    np.testing.assert_array_equal(b, np.full(100, 2.5))
    del b
    gc.collect()
    assert pool.in_use_bytes == 800 and not pool.free
    del a
    gc.collect()
    assert pool.in_use_bytes == 0 and len(pool.free) == 1
