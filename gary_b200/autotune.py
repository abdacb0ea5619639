"""Project autotuner: times the counting kernel over a grid of tile shapes
(target work per warp tile, per CTA tile) and resident CTAs per SM, on the
graph at hand, and keeps the fastest.  Knobs are the process-wide gary_tune
parameters; cached plans are dropped so each candidate rebuilds its tiles.

    best = autotune(graph, count_fn)   # count_fn() launches one count
"""
from __future__ import annotations

import itertools
import json

from ._lib import check, load

# warp_tile_cost 0 = the library's own sizing from the graph's work
GRID = {
    "warp_tile_cost": (0, 1 << 11, 1 << 13, 1 << 15),
    "cta_tile_cost": (1 << 18, 1 << 20),
    "min_blocks": (2, 3),
}


def apply(cfg: dict) -> None:
    L = load()
    check(L.gary_tune(b"reset", 0), "gary_tune")
    for k, v in cfg.items():
        check(L.gary_tune(k.encode(), int(v)), "gary_tune")


def autotune(graph, count_fn, grid: dict = GRID, reps: int = 3, log=None) -> dict:
    """Return {'config': best, 'ms': best_ms, 'trials': [...]} and leave the
    best configuration applied (and graph's plans rebuilt for it)."""
    import torch

    keys = list(grid)
    trials = []
    for vals in itertools.product(*(grid[k] for k in keys)):
        cfg = dict(zip(keys, vals))
        apply(cfg)
        load().gary_graph_drop_plans(graph.handle)
        count_fn()  # builds the plan
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            count_fn()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        trials.append({"config": cfg, "ms": ms})
        if log:
            log(json.dumps(trials[-1]))
    best = min(trials, key=lambda t: t["ms"])
    apply(best["config"])
    load().gary_graph_drop_plans(graph.handle)
    count_fn()
    torch.cuda.synchronize()
    return {"config": best["config"], "ms": best["ms"], "trials": trials}
