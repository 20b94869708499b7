"""Shared fixtures and helpers.

Tests marked ``gpu`` need a CUDA device and the built ``libpsierra_b200.so``; the
rest run on the CPU (oracle against golden vectors, host pattern logic, the C ABI
exports, host drivers with fake domains, gloo multi-process paths).
"""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device and the built CUDA library")


def pytest_collection_modifyitems(config, items):
    try:
        import torch

        has_cuda = torch.cuda.is_available()
    except Exception:  # pragma: no cover
        has_cuda = False
    if has_cuda:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


def golden(name: str) -> dict:
    with np.load(os.path.join(GOLDEN, f"{name}.npz"), allow_pickle=False) as z:
        return {k: z[k] for k in z.files}


def rel_max(a, ref) -> float:
    """max |a - ref| / max |ref|."""
    a = np.asarray(a, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    return float(np.abs(a - ref).max() / np.abs(ref).max())


def rel_2(a, ref) -> float:
    """||a - ref||_2 / ||ref||_2."""
    a = np.asarray(a, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    return float(np.linalg.norm(a - ref) / np.linalg.norm(ref))


def disjoint_mesh(X: np.ndarray):
    """Mesh whose elements share no nodes: element i owns nodes npe*i .. npe*i+npe-1."""
    from psierra_b200.meshgen import TetMesh

    n, npe, _ = X.shape
    return TetMesh(X.reshape(-1, 3).copy(), np.arange(n * npe, dtype=np.int64).reshape(n, npe))


def block_diagonal_blocks(K, n: int, d: int) -> np.ndarray:
    """(n, d, d) diagonal blocks of a block-diagonal sparse matrix."""
    Kd = K.toarray()
    return np.stack([Kd[d * i:d * i + d, d * i:d * i + d] for i in range(n)])
