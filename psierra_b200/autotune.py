"""Launch-shape autotuner of the persistent assembly kernel.

Two knobs change the speed of ``psx_tet4_assemble`` / ``psx_tet10_assemble`` on a given
mesh without changing a single output bit (each K and f entry is summed by one owner in
a fixed order whatever the schedule): the lag (granules between an element tile and the
gathers it completes, which trades L2-resident ring size for fewer waits) and the number
of persistent blocks per SM.  ``tune`` times each candidate with CUDA events on the
caller's stream and keeps the fastest; results are cached per device, element type,
mesh size and precision, in memory and optionally in a JSON file.
"""
from __future__ import annotations

import json
import os

import torch

DEFAULT_LAGS = (4, 8, 16)
DEFAULT_BLOCKS = (1, 2, 3)

_cache: dict[str, tuple[int, int]] = {}


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
    return a.elapsed_time(b) / reps


def tune(asm, u: torch.Tensor, precision: str | None = None, want_f: bool = True, want_k: bool = True,
         lags=DEFAULT_LAGS, blocks=DEFAULT_BLOCKS, reps: int = 5, cache_file: str | None = None) -> dict:
    """Pick (lag, blocks_per_sm) for ``asm`` by timing; applies and returns the choice.

    Returns ``{"lag", "blocks_per_sm", "ms", "table": {(lag, bps): ms}}``.  With a cached
    entry for the same key nothing is timed.
    """
    prec = precision or asm.precision
    key = _key(asm, prec, want_f, want_k)
    disk = {}
    if cache_file and os.path.exists(cache_file):
        with open(cache_file) as fh:
            disk = json.load(fh)
    hit = _cache.get(key) or (tuple(disk[key]) if key in disk else None)
    if hit is not None:
        asm.set_queue(lag=hit[0], blocks_per_sm=hit[1])
        return {"lag": hit[0], "blocks_per_sm": hit[1], "ms": None, "table": {}}
    f = asm.new_f() if want_f else None
    k = asm.new_k(prec) if want_k else None
    table = {}
    for lag in lags:
        for bps in blocks:
            asm.set_queue(lag=lag, blocks_per_sm=bps)
            table[(lag, bps)] = _time(asm, u, prec, want_f, want_k, f, k, reps)
    best = min(table, key=table.get)
    asm.set_queue(lag=best[0], blocks_per_sm=best[1])
    _cache[key] = best
    if cache_file:
        disk[key] = list(best)
        with open(cache_file, "w") as fh:
            json.dump(disk, fh, indent=1, sort_keys=True)
    return {"lag": best[0], "blocks_per_sm": best[1], "ms": table[best], "table": table}
