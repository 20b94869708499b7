"""Launch-shape autotuner of the persistent assembly kernel.

Three knobs change the speed of ``psx_tet4_assemble`` / ``psx_tet10_assemble`` on a given
mesh without changing a single output bit (each K and f entry is summed by one owner in
a fixed order whatever the schedule): the lag of the task queue in use (granules between
an element tile and the gathers it completes: too small and gathers wait for elements
still in flight, too large and the ring outgrows L2), the ring slack (room for element
tiles in flight before they must wait for old gathers), the number of persistent
blocks per SM and, for Tet4 FP32 tangent sweeps, whether element tiles and gathers run
in separate warps (the warp-specialised kernel, whose ring is sized by the same lag and
slack) or in the same ones.  ``tune`` times each candidate with CUDA events on the
caller's stream and keeps the fastest; results are cached per device, element type,
mesh size and precision, in memory and optionally in a JSON file.
"""
from __future__ import annotations

import json
import os

import torch

from psierra_b200.assembler import raise_if_wait_gave_up

DEFAULT_LAGS = (8, 12, 16, 24)
DEFAULT_BLOCKS = (2,)
DEFAULT_SLACKS = (6, 12, 20)

DEFAULT_SPLITS = (True, False)

_cache: dict[str, tuple] = {}


def _key(asm, precision: str, want_f: bool, want_k: bool) -> str:
    name = torch.cuda.get_device_name(asm.device)
    return f"{name}|npe{asm.npe}|E{asm.n_elements}|N{asm.n_nodes}|{precision}|f{int(want_f)}k{int(want_k)}"


def _time(asm, u, precision, want_f, want_k, f, k, reps: int) -> float:
    for _ in range(2):
        asm.assemble(u, want_f=want_f, want_k=want_k, precision=precision, f_out=f, k_out=k, check_status=False)
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        asm.assemble(u, want_f=want_f, want_k=want_k, precision=precision, f_out=f, k_out=k, check_status=False)
    b.record()
    b.synchronize()
    # the status of the last timed call: a candidate whose bounded wait gave up is not a
    # valid launch shape
    raise_if_wait_gave_up(asm.status_counts()[3])
    return a.elapsed_time(b) / reps


def _apply(asm, want_k: bool, lag: int, bps: int, slack: int, split: bool | None = None) -> None:
    if want_k:
        asm.set_queue(lag=lag, blocks_per_sm=bps, ring_slack=slack, split=split)
    else:
        asm.set_queue(lag_f=lag, blocks_per_sm=bps, ring_slack=slack)


def tune(asm, u: torch.Tensor, precision: str | None = None, want_f: bool = True, want_k: bool = True,
         lags=DEFAULT_LAGS, blocks=DEFAULT_BLOCKS, slacks=DEFAULT_SLACKS, splits=DEFAULT_SPLITS, reps: int = 5,
         cache_file: str | None = None) -> dict:
    """Pick (lag, blocks_per_sm, ring_slack, split) for ``asm`` by timing; applies and returns it.

    The lag tuned is that of the queue the sweep uses (the K queue when ``want_k``, else
    the f queue).  ``splits`` is swept only for Tet4 FP32 tangent sweeps (the only ones
    with a warp-specialised kernel); elsewhere split is left as it is.  Returns
    ``{"lag", "blocks_per_sm", "ring_slack", "split", "ms", "table": {(lag, bps, slack,
    split): ms}}``.  With a cached entry for the same key nothing is timed.
    """
    prec = precision or asm.precision
    key = _key(asm, prec, want_f, want_k)
    disk = {}
    if cache_file and os.path.exists(cache_file):
        with open(cache_file) as fh:
            disk = json.load(fh)
    hit = _cache.get(key) or (tuple(disk[key]) if key in disk else None)
    if hit is not None:
        hit = tuple(hit) + (asm.pattern.split,) * (4 - len(hit))
        _apply(asm, want_k, *hit)
        return {"lag": hit[0], "blocks_per_sm": hit[1], "ring_slack": hit[2], "split": hit[3], "ms": None,
                "table": {}}
    f = asm.new_f() if want_f else None
    k = asm.new_k(prec) if want_k else None
    has_split = asm.npe == 4 and want_k and prec == "fp32-mixed"
    split_opts = tuple(bool(x) for x in splits) if has_split else (asm.pattern.split,)
    table = {}
    for split in split_opts:
        for lag in lags:
            for bps in blocks:
                for slack in slacks:
                    _apply(asm, want_k, lag, bps, slack, split)
                    table[(lag, bps, slack, split)] = _time(asm, u, prec, want_f, want_k, f, k, reps)
    best = min(table, key=table.get)
    _apply(asm, want_k, *best)
    _cache[key] = best
    if cache_file:
        disk[key] = list(best)
        with open(cache_file, "w") as fh:
            json.dump(disk, fh, indent=1, sort_keys=True)
    return {"lag": best[0], "blocks_per_sm": best[1], "ring_slack": best[2], "split": best[3], "ms": table[best],
            "table": table}
