"""Autotuner for the wavefront renderer.

The wavefront mode's throughput depends on knobs that never change a result:
  * the path-slot pool (how many paths are in flight: latency hiding against working-set size)
    and how many samples a pass holds before they are folded into the images (tune_wavefront);
  * the compiled kernel variants and thresholds (tune_kernels): the traversal kernels' block
    shape (192 x 6, 128 x 9 or 256 x 4 threads x blocks per SM), the surface-shading block
    (512 or 256 threads), how many idle lanes a closest-hit or shadow traversal warp gathers
    before it takes new rays from the queue, and whether shadow rays walk a 4-wide view of the
    BVHs.
The tuner times a representative call for each candidate on the renderer's own stream (CUDA
events, after one warm-up call) and keeps the fastest; tune_kernels does it one knob at a time
(coordinate descent: each knob swept with the others at their current best).  The chosen
configuration and the full timing tables are returned for the caller to record.
"""
from __future__ import annotations

from typing import Callable, Iterable

POOL_CANDIDATES = (1 << 23, 1 << 24, 1 << 25, 1 << 26)
UNITS_CANDIDATES = (1 << 27, 1 << 29)


def time_call(renderer, fn: Callable[[], object], repeats: int = 1) -> float:
    """Device milliseconds of fn() on the renderer's stream (mean over `repeats`, after a warm-up)."""
    import torch
    stream = torch.cuda.ExternalStream(renderer.stream_handle())
    fn()
    renderer.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(repeats):
        fn()
    e1.record(stream)
    renderer.synchronize()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / repeats


def tune_wavefront(renderer, fn: Callable[[], object], pools: Iterable[int] = POOL_CANDIDATES,
                   units: Iterable[int] = UNITS_CANDIDATES, repeats: int = 1, timer=None) -> dict:
    """Times fn() for every (pool, units_per_pass) pair, applies the fastest and returns
    {"pool_paths", "units_per_pass", "ms", "table": [(pool, units, ms), ...]}.  `timer(renderer,
    fn, repeats)` defaults to time_call (CUDA events on the renderer's stream); ties keep the
    first candidate in table order."""
    timer = timer or time_call
    table = []
    for u in units:
        for p in pools:
            renderer.set_wavefront_config(p, u)
            table.append((p, u, timer(renderer, fn, repeats)))
    best = min(table, key=lambda row: row[2])
    renderer.set_wavefront_config(best[0], best[1])
    return {"pool_paths": best[0], "units_per_pass": best[1], "ms": best[2], "table": table}


TRAV_SHAPES = {0: "192x6", 1: "128x9", 2: "256x4"}
KERNEL_KNOBS = (
    ("shadow_wide", (1, 0)),
    ("trav_shape", (0, 1, 2)),
    ("refill_closest", (8, 16, 24, 28)),
    ("refill_shadow", (4, 8, 16)),
    ("shade_block", (512, 256)),
)


def tune_kernels(renderer, fn: Callable[[], object], knobs=KERNEL_KNOBS, repeats: int = 1, timer=None) -> dict:
    """Coordinate descent over the wavefront kernel variants: starting from the renderer's
    current tuning, each knob in turn is swept over its candidates (the others held at their
    best so far) and set to its fastest value.  Returns {"tuning": {...}, "ms": best time,
    "table": {knob: [(value, ms), ...]}}; ties keep the earlier candidate."""
    timer = timer or time_call
    cur = dict(renderer.wavefront_tuning())
    tables = {}
    best_ms = None
    for name, cands in knobs:
        rows = []
        for v in cands:
            trial = dict(cur)
            trial[name] = v
            renderer.set_wavefront_tuning(**trial)
            rows.append((v, timer(renderer, fn, repeats)))
        v_best, ms = min(rows, key=lambda row: row[1])
        cur[name] = v_best
        best_ms = ms
        tables[name] = rows
    renderer.set_wavefront_tuning(**cur)
    return {"tuning": cur, "ms": best_ms, "table": tables}
