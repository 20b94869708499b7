"""Deadlock freedom and ring safety of the persistent assembly kernel's task queue (CPU).

The kernel's wait rules, restated:
* gather tiles of granule r are queued after the element tiles of granule r + 1 + lag;
* an element tile of granule g waits for all gather tiles of granules
  [g - R, g - R + span_g + 1] (R = ring length in granules) before overwriting the ring
  slots of granule g - R, if g - R >= 0;
* a gather tile of granule r waits for all element tiles of granules [r - span_g - 1, r].
The warp-specialised kernel's loops wait on prefixes instead ([0, g - R + span_g + 1] and
[0, r]: each warp keeps a watermark of the granules it knows are complete), which contain
those spans.
Tasks are claimed in queue order by running blocks, so the queue always drains if every
task only waits on tasks strictly earlier in the queue.  Ring safety: every gather item
that reads an element of granule q belongs to a granule in [q, q + span_g + 1].
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from psierra_b200 import _lib, meshgen
from psierra_b200.pattern import MeshPattern


def _queue(p: MeshPattern, with_pairs: int, tile: int, lag: int):
    h = p.plan_host()
    st = _lib.PlanStruct()
    st.npe, st.n_granules = p.npe, h["n_granules"]
    st.n_elements, st.n_nodes, st.n_pairs = p.n_elements, p.n_nodes, h["n_pairs"]
    st.granule, st.max_span = p.granule, int(h["max_span"][0])
    st.pair_gptr, st.node_gptr = h["pair_gptr"].ctypes.data, h["node_gptr"].ctypes.data
    L = _lib.lib()
    nt = ctypes.c_int64()
    _lib.check(L.psx_task_count(ctypes.byref(st), with_pairs, tile, tile, lag, ctypes.byref(nt)), "count")
    tasks = np.zeros(4 * nt.value, dtype=np.int32)
    bt = np.zeros(h["n_granules"], dtype=np.int32)
    _lib.check(L.psx_task_fill(ctypes.byref(st), with_pairs, tile, tile, lag, _lib.ptr(tasks), _lib.ptr(bt)), "fill")
    return tasks.reshape(-1, 4), bt, h


@pytest.mark.parametrize("granule,with_pairs,lag", [(256, 1, 0), (256, 0, 4), (512, 1, 4), (128, 1, 2),
                                                    (128, 1, 7)])
def test_waits_only_on_earlier_tasks(granule, with_pairs, lag):
    m = meshgen.box_tet4(1.0, 1.0, 1.0, 9, 8, 7)
    p = MeshPattern(m.elements, m.n_nodes)
    p.granule = granule
    tile = 64
    tasks, bt, h = _queue(p, with_pairs, tile, lag)
    G = h["n_granules"]
    span_g = -(-int(h["max_span"][0]) // granule)
    # all items covered exactly once
    kinds = tasks[:, 0]
    assert tasks[kinds == 0, 3].sum() - tasks[kinds == 0, 2].sum() == m.n_elements
    assert tasks[kinds == 2, 3].sum() - tasks[kinds == 2, 2].sum() == m.n_nodes
    if with_pairs:
        assert tasks[kinds == 1, 3].sum() - tasks[kinds == 1, 2].sum() == h["n_pairs"]
    # gather tile counts per granule match
    for r in range(G):
        assert bt[r] == np.count_nonzero((kinds != 0) & (tasks[:, 1] == r))
    # the kernel's ring length (power of two >= span_g + lag + 6, capped to cover all granules)
    all_g = 1 << int(np.ceil(np.log2(max(G, 1))))
    ring = 1 << int(np.ceil(np.log2(span_g + lag + 6)))
    ring = min(ring, all_g)
    last_a = {}
    last_b = {}
    for q, (kind, g, b, e) in enumerate(tasks):
        if kind == 0:
            last_a[g] = q
        else:
            last_b[g] = q
    first_pos = {}
    for q, (kind, g, b, e) in enumerate(tasks):
        first_pos.setdefault((kind == 0, g), q)
    for q, (kind, g, b, e) in enumerate(tasks):
        if kind == 0:
            old = g - ring
            if old >= 0:
                for r in range(old, min(old + span_g + 2, G)):
                    assert last_b.get(r, -1) < q, "element tile waits on a later gather tile"
        else:
            for gp in range(max(0, g - span_g - 1), g + 1):
                assert last_a[gp] < q, "gather tile waits on a later element tile"
    # ring safety: items read elements within span_g + 1 granules of their own granule
    for kind, g, b, e in tasks[kinds != 0]:
        if kind == 1:
            srcs = h["pair_src"][h["pair_ptr"][b]:h["pair_ptr"][e]] >> 6
        else:
            srcs = h["node_src"][h["node_ptr"][b]:h["node_ptr"][e]] >> 4
        if srcs.size:
            assert (srcs // granule).min() >= g - span_g - 1 and (srcs // granule).max() <= g


@pytest.mark.parametrize("granule,lag,workers,seed", [(128, 0, (1, 1), 0), (128, 2, (3, 2), 1), (256, 4, (2, 5), 2),
                                                      (64, 0, (4, 4), 3)])
def test_split_queues_drain(granule, lag, workers, seed):
    """The warp-specialised kernel's two queues: element tiles claimed in index order by
    element warps, the gather tasks of the K queue claimed in order by gather warps, with
    the same waits.  A random schedule of a few workers per role must always drain, and
    a gather tile may only run once every element tile of its span is done."""
    m = meshgen.box_tet4(1.0, 1.0, 1.0, 9, 8, 7)
    p = MeshPattern(m.elements, m.n_nodes)
    p.granule = granule
    tile = 32
    tasks, bt, h = _queue(p, 1, tile, lag)
    G = h["n_granules"]
    span_g = -(-int(h["max_span"][0]) // granule)
    all_g = 1 << int(np.ceil(np.log2(max(G, 1))))
    ring = min(1 << int(np.ceil(np.log2(span_g + lag + 6))), all_g)
    n_tiles = -(-m.n_elements // tile)
    gtasks = tasks[tasks[:, 0] != 0]
    atiles = [-(-min(granule, m.n_elements - r * granule) // tile) for r in range(G)]
    done_a = np.zeros(G, dtype=np.int64)
    done_b = np.zeros(G, dtype=np.int64)
    nxt = {"e": 0, "g": 0}
    held = {("e", i): None for i in range(workers[0])}
    held.update({("g", i): None for i in range(workers[1])})
    rng = np.random.default_rng(seed)

    def ready(role, t):
        if role == "e":
            old = t * tile // granule - ring
            return old < 0 or all(done_b[r] >= bt[r] for r in range(0, min(old + span_g + 2, G)))
        g = gtasks[t, 1]
        return all(done_a[r] >= atiles[r] for r in range(0, g + 1))

    remaining = n_tiles + len(gtasks)
    while remaining:
        moves = []
        for w, t in held.items():
            role = w[0]
            if t is None:
                if nxt[role] < (n_tiles if role == "e" else len(gtasks)):
                    moves.append(w)
            elif ready(role, t):
                moves.append(w)
        assert moves, "split queues deadlocked"
        w = moves[rng.integers(len(moves))]
        role, t = w[0], held[w]
        if t is None:
            held[w] = nxt[role]
            nxt[role] += 1
        else:
            if role == "e":
                done_a[t * tile // granule] += 1
            else:
                g = gtasks[t, 1]
                # everything this gather tile reads is complete
                assert all(done_a[r] >= atiles[r] for r in range(max(0, g - span_g - 1), g + 1))
                done_b[g] += 1
            held[w] = None
            remaining -= 1
    assert (done_a == np.array(atiles)).all() and (done_b == bt).all()


def test_split_plan_lists_the_gather_tasks_in_queue_order():
    """The plan's gather-only list (psx_plan_t.gtasks_k) is the K queue without its element
    tiles, in queue order; switching the split off clears it (the mixed kernel runs)."""
    m = meshgen.box_tet4(1.0, 1.0, 1.0, 6, 5, 4)
    p = MeshPattern(m.elements, m.n_nodes)
    d = p.device("cpu")
    st = d["plan"]
    tasks = d["tasks_k"].numpy().reshape(-1, 4)[: st.n_tasks_k]
    gk = d["gtasks_k"].numpy().reshape(-1, 4)
    assert np.array_equal(gk, tasks[tasks[:, 0] != 0])
    assert st.n_gtasks_k == len(gk) and st.gtasks_k == d["gtasks_k"].data_ptr()
    # element tiles are implicit in the split kernel: consecutive 32-element tiles
    et = tasks[tasks[:, 0] == 0]
    assert np.array_equal(et[:, 2], np.arange(len(et)) * p.tile)
    assert np.array_equal(et[:, 1], et[:, 2] // p.granule)
    p.set_queue(split=False)
    assert st.n_gtasks_k == 0 and not st.gtasks_k
    p.set_queue(split=True)
    assert st.n_gtasks_k == len(gk) and st.gtasks_k == d["gtasks_k"].data_ptr()
    # the lag changes the K queue's interleaving, not its gather order
    p.set_queue(lag=3)
    d2 = p.device("cpu")
    assert np.array_equal(d2["gtasks_k"].numpy().reshape(-1, 4), gk)


@pytest.mark.parametrize("granule,lag,workers,seed", [(128, 0, (1, 1), 4), (128, 2, (3, 2), 5), (64, 0, (4, 4), 6),
                                                      (64, 1, (2, 1), 7)])
def test_split_queues_drain_with_deferred_publish(granule, lag, workers, seed):
    """Element warps claim tiles two ahead (they hold the tile they work on and the next
    one) and publish a finished tile only once their next tile has been evaluated, or
    earlier when that next tile's ring wait is not yet satisfied (psx_gather.cuh
    drain_elements).  Waits are on prefixes.  A random schedule must still drain."""
    m = meshgen.box_tet4(1.0, 1.0, 1.0, 9, 8, 7)
    p = MeshPattern(m.elements, m.n_nodes)
    p.granule = granule
    tile = 32
    tasks, bt, h = _queue(p, 1, tile, lag)
    G = h["n_granules"]
    span_g = -(-int(h["max_span"][0]) // granule)
    all_g = 1 << int(np.ceil(np.log2(max(G, 1))))
    ring = min(1 << int(np.ceil(np.log2(span_g + lag + 6))), all_g)
    n_tiles = -(-m.n_elements // tile)
    gtasks = tasks[tasks[:, 0] != 0]
    atiles = [-(-min(granule, m.n_elements - r * granule) // tile) for r in range(G)]
    done_a = np.zeros(G, dtype=np.int64)
    done_b = np.zeros(G, dtype=np.int64)
    rng = np.random.default_rng(seed)
    nxt = {"e": 0, "g": 0}
    # element worker: [claimed tiles (at most two, the first is worked on), evaluated?,
    # pending (finished, unpublished) tile or None]
    ew = [[[], False, None] for _ in range(workers[0])]
    gw = [None] * workers[1]

    def e_ready(t):
        old = t * tile // granule - ring
        return old < 0 or all(done_b[r] >= bt[r] for r in range(0, min(old + span_g + 2, G)))

    def g_ready(t):
        return all(done_a[r] >= atiles[r] for r in range(0, gtasks[t, 1] + 1))

    def publish(w):
        if w[2] is not None:
            done_a[w[2] * tile // granule] += 1
            w[2] = None

    remaining = n_tiles + len(gtasks)
    while remaining or any(w[2] is not None for w in ew):
        moves = []
        for i, w in enumerate(ew):
            if len(w[0]) < 2 and nxt["e"] < n_tiles:
                moves.append(("claim_e", i))
            if not w[0]:
                if nxt["e"] >= n_tiles and w[2] is not None:
                    moves.append(("flush", i))  # the queue is empty: publish and leave
            elif not w[1]:
                if e_ready(w[0][0]):
                    moves.append(("eval", i))
                elif w[2] is not None:
                    moves.append(("flush", i))  # about to block: publish first
            else:
                moves.append(("finish", i))
        for i, t in enumerate(gw):
            if t is None:
                if nxt["g"] < len(gtasks):
                    moves.append(("claim_g", i))
            elif g_ready(t):
                moves.append(("gather", i))
        assert moves, "split queues deadlocked"
        kind, i = moves[rng.integers(len(moves))]
        if kind == "claim_e":
            ew[i][0].append(nxt["e"])
            nxt["e"] += 1
        elif kind == "flush":
            publish(ew[i])
        elif kind == "eval":
            ew[i][1] = True
            publish(ew[i])  # the previous tile goes out after this tile's evaluation
        elif kind == "finish":
            ew[i][2], ew[i][1] = ew[i][0].pop(0), False
            remaining -= 1
        elif kind == "claim_g":
            gw[i] = nxt["g"]
            nxt["g"] += 1
        else:
            t = gw[i]
            g = gtasks[t, 1]
            assert all(done_a[r] >= atiles[r] for r in range(max(0, g - span_g - 1), g + 1))
            done_b[g] += 1
            gw[i] = None
            remaining -= 1
    assert (done_a == np.array(atiles)).all() and (done_b == bt).all()
