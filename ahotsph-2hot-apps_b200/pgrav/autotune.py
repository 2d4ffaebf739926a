"""Autotuner of the batched kernels' tile shapes.

The search space is grav_tuning: warps per block (4 or 8), resident blocks
per SM (0 = as many as registers and shared memory allow, or a cap), the
list-chunk length of each kind (the work-item size; the automatic choice
times a scale) and, for periodic plans, where the Ewald correction moments
run (a side stream beside the list kernels, or the finish pass).  Each
candidate is applied with grav_plan_retune_CUDA, which rebuilds only the
work queue, and timed with CUDA events over a few evaluations; the search
is coordinate-wise (launch shape, then chunk scale, then the moments'
placement) and leaves the plan on the best shape.
"""
import json
import os

import numpy as np

from . import gravcuda as gc

TILE = 32


def _time(plan, stream, reps):
    import torch
    plan.eval(stream.cuda_stream)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(reps):
        plan.eval(stream.cuda_stream)
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def _scaled(base, s):
    return int(max(TILE, round(base * s / TILE) * TILE))


def autotune(plan, reps=3, shapes=((8, 0), (4, 0), (8, 1), (8, 2), (4, 2), (4, 4)),
             scales=(0.25, 0.5, 1.0, 2.0, 4.0), sides=(-2, -4, 2, 3), cache=None, key=None):
    """Tune `plan` in place.  Returns (best gc.Tuning, list of trials).  With
    `cache` (a JSON file path) and `key`, a stored result is applied without
    a search, and a new one is stored."""
    import torch
    if cache and key and os.path.exists(cache):
        table = json.load(open(cache))
        if key in table:
            t = gc.Tuning(*table[key]["tuning"])
            plan.retune(t)
            return plan.tuning(), table[key]["trials"]
    stream = torch.cuda.Stream()
    base = plan.tuning()
    base_chunks = (base.chunk_p, base.chunk_q, base.chunk_h)
    trials = []

    def trial(wpb, bps, s, side=0):
        t = gc.Tuning(wpb, _scaled(base_chunks[0], s), _scaled(base_chunks[1], s),
                      _scaled(base_chunks[2], s), bps, base.ewald_n, side)
        plan.retune(t)
        ms = _time(plan, stream, reps)
        trials.append({"warps_per_block": wpb, "blocks_per_sm": bps, "chunk_scale": s,
                       "chunks": [t.chunk_p, t.chunk_q, t.chunk_h], "ewald_side": side, "ms": ms})
        return ms

    best = min(((trial(w, b, 1.0), w, b) for w, b in shapes))
    _, wpb, bps = best
    best_s = min(((trial(wpb, bps, s), s) for s in scales if s != 1.0), default=(best[0], 1.0))
    s = best_s[1] if best_s[0] < best[0] else 1.0
    best_ms = min(best[0], best_s[0])
    side = 0
    if getattr(plan, "ewald", False) and sides:
        best_side = min(((trial(wpb, bps, s, sd), sd) for sd in sides), default=(best_ms, 0))
        side = best_side[1] if best_side[0] < best_ms else 0
    t = gc.Tuning(wpb, _scaled(base_chunks[0], s), _scaled(base_chunks[1], s),
                  _scaled(base_chunks[2], s), bps, base.ewald_n, side)
    plan.retune(t)
    if cache and key:
        table = json.load(open(cache)) if os.path.exists(cache) else {}
        table[key] = {"tuning": [t.warps_per_block, t.chunk_p, t.chunk_q, t.chunk_h,
                                 t.blocks_per_sm, t.ewald_n, t.ewald_side], "trials": trials}
        with open(cache, "w") as f:
            json.dump(table, f, indent=1)
    return plan.tuning(), trials


def signature(tree):
    """A cache key for problems of the same shape: sizes and list lengths."""
    c = np.asarray(tree.counts, np.float64) / max(tree.n, 1)
    return (f"n{int(np.log2(max(tree.n, 1)))}-g{int(np.log2(max(tree.ngroups, 1)))}-"
            + "-".join(f"{int(round(np.log2(1 + x) * 4))}" for x in c))
