"""Autotuner bookkeeping (CPU, with a fake assembler and fake timings): the fastest
candidate is applied and returned, results are cached per device / element type / mesh
size / precision / sweep in memory and in a JSON file, a cached entry is applied without
timing anything, and the split option is swept only for Tet4 FP32 tangent sweeps."""
from __future__ import annotations

import json
import types

import pytest
import torch

from psierra_b200 import autotune


class FakeAssembler:
    def __init__(self, npe=4, precision="fp32-mixed"):
        self.device = torch.device("cpu")
        self.npe, self.n_elements, self.n_nodes, self.precision = npe, 1000, 300, precision
        self.pattern = types.SimpleNamespace(split=npe == 4)
        self.applied = []

    def set_queue(self, lag=None, blocks_per_sm=None, ring_slack=None, lag_f=None, split=None):
        self.applied.append({"lag": lag, "lag_f": lag_f, "bps": blocks_per_sm, "slack": ring_slack, "split": split})

    def new_f(self):
        return None

    def new_k(self, prec):
        return None


@pytest.fixture
def fake_timing(monkeypatch):
    timed = []

    def fake_time(asm, u, prec, want_f, want_k, f, k, reps):
        cfg = asm.applied[-1]
        lag = cfg["lag"] if want_k else cfg["lag_f"]
        timed.append((lag, cfg["slack"], cfg["split"]))
        # fastest at lag 16, slack 12, split on
        return abs(lag - 16) + 0.1 * abs(cfg["slack"] - 12) + (0.0 if cfg["split"] in (True, None) else 5.0)

    monkeypatch.setattr(autotune, "_time", fake_time)
    monkeypatch.setattr(torch.cuda, "get_device_name", lambda *a, **k: "FakeGPU")
    monkeypatch.setattr(autotune, "_cache", {})
    return timed


def test_fastest_candidate_is_applied_and_cached(fake_timing, tmp_path):
    asm = FakeAssembler()
    cache = tmp_path / "tune.json"
    r = autotune.tune(asm, None, lags=(8, 16, 24), slacks=(6, 12), cache_file=str(cache))
    assert (r["lag"], r["ring_slack"], r["split"]) == (16, 12, True)
    assert len(fake_timing) == 3 * 2 * 2  # lags x slacks x split on/off for the Tet4 FP32 tangent
    assert asm.applied[-1]["lag"] == 16 and asm.applied[-1]["slack"] == 12 and asm.applied[-1]["split"] is True
    disk = json.loads(cache.read_text())
    (key, val), = disk.items()
    assert key.startswith("FakeGPU|npe4|E1000|N300|fp32-mixed|f1k1") and val[0] == 16 and val[2] == 12

    # same key again: nothing is timed, the cached shape is applied
    fake_timing.clear()
    asm2 = FakeAssembler()
    r2 = autotune.tune(asm2, None, lags=(8, 16, 24), slacks=(6, 12), cache_file=str(cache))
    assert fake_timing == [] and r2["ms"] is None and r2["lag"] == 16
    assert asm2.applied == [{"lag": 16, "lag_f": None, "bps": r["blocks_per_sm"], "slack": 12, "split": True}]

    # a fresh process (empty memory cache) reads the file
    autotune._cache.clear()
    asm3 = FakeAssembler()
    r3 = autotune.tune(asm3, None, cache_file=str(cache))
    assert fake_timing == [] and r3["lag"] == 16 and asm3.applied[-1]["slack"] == 12


def test_sweeps_without_a_tangent_tune_the_f_queue_and_not_the_split(fake_timing):
    asm = FakeAssembler()
    r = autotune.tune(asm, None, want_k=False, lags=(12, 16), slacks=(12,))
    assert r["lag"] == 16 and len(fake_timing) == 2
    assert all(a["lag"] is None and a["lag_f"] in (12, 16) for a in asm.applied)
    assert {t[2] for t in fake_timing} == {None}


@pytest.mark.parametrize("npe, prec", [(10, "fp32-mixed"), (4, "fp64")])
def test_split_is_not_swept_outside_tet4_fp32_tangent(fake_timing, npe, prec):
    asm = FakeAssembler(npe=npe, precision=prec)
    autotune.tune(asm, None, lags=(16,), slacks=(12,))
    assert len(fake_timing) == 1 and fake_timing[0][2] == asm.pattern.split
