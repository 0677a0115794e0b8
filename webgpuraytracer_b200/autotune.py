"""Autotuner for the wavefront renderer's sizing.

The wavefront mode's throughput depends on the path-slot pool (how many paths are in flight:
latency hiding against working-set size) and on how many samples a pass holds before they are
folded into the images (pass count against sample-buffer memory).  Neither changes a result, so
the tuner simply times a representative call for each candidate on the renderer's own stream
(CUDA events, after one warm-up call) and keeps the fastest.  The chosen configuration and the
full timing table are returned for the caller to record.
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
