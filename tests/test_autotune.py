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


class FakeTunable:
    """Stand-in renderer with the kernel-variant tuning interface."""

    def __init__(self):
        self.t = {"trav_shape": 0, "shade_block": 512, "refill_closest": 24, "refill_shadow": 8, "shadow_wide": 1}
        self.history = []

    def wavefront_tuning(self):
        return dict(self.t)

    def set_wavefront_tuning(self, **t):
        self.t = dict(t)
        self.history.append(dict(t))


def test_kernel_tuning_is_coordinate_descent():
    """Each knob is swept with the earlier knobs at their best and the later ones at their
    starting values; the best of every sweep is kept and the final tuning is left applied."""
    def cost(t):
        c = {0: 10.0, 1: 9.0, 2: 12.0}[t["trav_shape"]]
        c += {8: 1.0, 16: 0.5, 24: 0.7, 28: 0.9}[t["refill_closest"]] * (2.0 if t["trav_shape"] == 1 else 1.0)
        c += {4: 0.3, 8: 0.2, 16: 0.4}[t["refill_shadow"]]
        c += {512: 0.0, 256: 0.1}[t["shade_block"]]
        c += {1: 0.0, 0: 0.5}[t["shadow_wide"]]
        return c

    r = FakeTunable()
    out = autotune.tune_kernels(r, lambda: None, timer=lambda rr, fn, rep: cost(rr.t))
    assert out["tuning"] == {"trav_shape": 1, "shade_block": 512, "refill_closest": 16, "refill_shadow": 8,
                             "shadow_wide": 1}
    assert r.t == out["tuning"]
    assert [v for v, _ in out["table"]["trav_shape"]] == [0, 1, 2]
    # the refill sweep ran with the chosen shape (1), so its costs are doubled
    assert dict(out["table"]["refill_closest"])[16] == cost({**out["tuning"], "refill_shadow": 8, "refill_closest": 16})
    assert len(r.history) == 2 + 3 + 4 + 3 + 2 + 1
    assert out["ms"] == min(ms for _, ms in out["table"]["shade_block"])


def test_kernel_knob_candidates_are_valid():
    knobs = dict(autotune.KERNEL_KNOBS)
    assert set(knobs["trav_shape"]) <= {0, 1, 2}
    assert set(knobs["shade_block"]) <= {256, 512}
    assert set(knobs["shadow_wide"]) <= {0, 1}
    assert all(1 <= v <= 32 for v in knobs["refill_closest"] + knobs["refill_shadow"])
