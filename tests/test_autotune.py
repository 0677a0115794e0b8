"""The wavefront autotuner's host logic with a stand-in renderer and timer (no GPU): every
(pool, units per pass) candidate is configured and timed once, in table order, and the fastest
configuration is left applied."""
from __future__ import annotations

from webgpuraytracer_b200 import autotune


class FakeRenderer:
    def __init__(self):
        self.config = None
        self.history = []

    def set_wavefront_config(self, pool, units):
        self.config = (pool, units)
        self.history.append((pool, units))


def _timer(costs):
    def timer(renderer, fn, repeats):
        fn()
        return costs[renderer.config]
    return timer


def test_fastest_configuration_is_applied():
    pools, units = (1 << 23, 1 << 24, 1 << 26), (1 << 27, 1 << 30)
    costs = {(p, u): 100.0 - 10 * i - j for j, u in enumerate(units) for i, p in enumerate(pools)}
    costs[(1 << 24, 1 << 30)] = 5.0
    calls = []
    r = FakeRenderer()
    out = autotune.tune_wavefront(r, lambda: calls.append(r.config), pools=pools, units=units,
                                  timer=_timer(costs))
    assert out["pool_paths"] == 1 << 24 and out["units_per_pass"] == 1 << 30 and out["ms"] == 5.0
    assert r.config == (1 << 24, 1 << 30)                       # left applied
    order = [(p, u) for u in units for p in pools]
    assert [row[:2] for row in out["table"]] == order           # units outer, pools inner
    assert r.history[:-1] == order and calls == order


def test_ties_keep_the_first_candidate():
    pools, units = (1 << 23, 1 << 24), (1 << 27,)
    r = FakeRenderer()
    out = autotune.tune_wavefront(r, lambda: None, pools=pools, units=units,
                                  timer=_timer({(p, u): 7.0 for p in pools for u in units}))
    assert (out["pool_paths"], out["units_per_pass"]) == (1 << 23, 1 << 27)


def test_default_candidates_are_valid_pool_sizes():
    assert all(1024 <= p <= 1 << 26 for p in autotune.POOL_CANDIDATES)
    assert all((1 << 16) <= u <= (1 << 30) for u in autotune.UNITS_CANDIDATES)
