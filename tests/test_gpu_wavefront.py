"""The wavefront renderer's scheduling does not change its results.

Every (sample, pixel) of a render call is a work unit; a pool of path slots traces the units and
starts a new one in a slot as soon as its path ends, and each pixel's samples are folded into
the running mean in sample order at the end.  Pool size, passes, the host-driven loop used for
stage timing and the graph-driven loop must therefore all give the reference's frame-by-frame
result bit for bit.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from webgpuraytracer_b200 import renderer as rd
from webgpuraytracer_b200 import scene as sc
from webgpuraytracer_b200 import synth
from webgpuraytracer_b200._lib import WgptError

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def flagship():
    s = synth.flagship_scene(1, 1920, 1080, 8)
    return s, sc.pack_scene_data(s)


def _params(scene, packed, w, h, frame=0, seed=1, section=(0, 0)):
    scene.camera.aspect = w / h
    scene.camera.update_rays2()
    return sc.pack_params(scene, packed, w, h, frame, seed, section)


def _oracle(packed, params, w, h, first, reps, sec):
    acc = np.zeros((h, w, 4), np.float32)
    out = np.zeros((h, w, 4), np.uint8)
    assert oracle.render(oracle.OracleScene(packed), params, first, reps, sec, acc, out,
                         oracle.default_threads()) == 0
    return acc, out


def _gpu(r, params, first, reps, sec):
    r._check(r.L.wgpt_set_params(r.ctx, rd.ptr(params)), "set_params")
    r._check(r.L.wgpt_render(r.ctx, first, reps, *sec), "render")
    r.synchronize()
    return r.read_accum(), r.read_output()


def _same(a, b, what):
    bad = ~((a == b) | (np.isnan(a) & np.isnan(b)))
    assert int(bad.sum()) == 0, f"{what}: {int(bad.sum())} values differ, first at {np.argwhere(bad)[:4].tolist()}"


def test_small_pool_and_several_passes_match_oracle(flagship):
    """1,024 path slots for 98,304 units (heavy regeneration) and a 65,536-unit pass limit (the
    8 samples run as passes of 5 and 3) still give the oracle's image bit for bit."""
    scene, packed = flagship
    w, h = 1920, 1080
    sec = (900, 500, 128, 96)
    params = _params(scene, packed, w, h, section=sec[:2])
    acc_o, out_o = _oracle(packed, params, w, h, 3, 8, sec)
    r = rd.Renderer(w, h)
    r.set_scene(scene, packed=packed)
    r.set_wavefront_config(1024, 65536)
    assert r.wavefront_config() == (1024, 65536)
    acc_g, out_g = _gpu(r, params, 3, 8, sec)
    ys, xs = slice(500, 596), slice(900, 1028)
    _same(acc_g[ys, xs], acc_o[ys, xs], "accumulation")
    _same(out_g[ys, xs], out_o[ys, xs], "rgba8")
    r.close()


def test_host_loop_equals_graph_loop(flagship):
    """Stage timing drives the iteration loop from the host with an event pair per launch; the
    result equals the graph-driven loop, and every stage reports launches."""
    scene, packed = flagship
    w, h = 1920, 1080
    sec = (400, 300, 256, 128)
    params = _params(scene, packed, w, h, section=sec[:2])
    r = rd.Renderer(w, h)
    r.set_scene(scene, packed=packed)
    acc_a, out_a = _gpu(r, params, 0, 4, sec)
    r.resize()
    r._check(r.L.wgpt_set_stage_timing(r.ctx, 1), "stage timing")
    acc_b, out_b = _gpu(r, params, 0, 4, sec)
    ms = np.zeros(8, np.float64)
    n = np.zeros(8, np.uint32)
    r._check(r.L.wgpt_read_stage_times(r.ctx, rd.ptr(ms), rd.ptr(n)), "stage times")
    r._check(r.L.wgpt_set_stage_timing(r.ctx, 0), "stage timing")
    _same(acc_a, acc_b, "accumulation")
    _same(out_a, out_b, "rgba8")
    assert n[0] == 1 and n[6] == 1                 # one fill and one accumulation per pass
    assert n[1] == n[2] == n[3] == n[4] == n[5] == n[7] >= 2   # one launch per stage per iteration
    assert np.all(ms[:8] > 0)
    r.close()


def test_one_call_equals_frame_by_frame(flagship):
    """render(reps=6) in one call equals six one-sample calls (sample_number 7..12)."""
    scene, packed = flagship
    w, h = 1920, 1080
    sec = (1200, 200, 160, 80)
    params = _params(scene, packed, w, h, section=sec[:2])
    r = rd.Renderer(w, h)
    r.set_scene(scene, packed=packed)
    acc_a, out_a = _gpu(r, params, 7, 6, sec)
    r.resize()
    for f in range(7, 13):
        acc_b, out_b = _gpu(r, params, f, 1, sec)
    _same(acc_a, acc_b, "accumulation")
    _same(out_a, out_b, "rgba8")
    r.close()


def test_zero_bounce_limit_matches_oracle():
    """BOUNCE_LIMIT = 0: the bounce loop never runs and every sample adds zero radiance."""
    s = synth.small_scene(1, 64, 64, 0)
    packed = sc.pack_scene_data(s)
    params = _params(s, packed, 64, 64)
    acc_o, out_o = _oracle(packed, params, 64, 64, 0, 3, (0, 0, 64, 64))
    for mode in (0, 1):
        r = rd.Renderer(64, 64)
        r.set_scene(s, packed=packed)
        r.set_render_mode(mode)
        acc_g, out_g = _gpu(r, params, 0, 3, (0, 0, 64, 64))
        _same(acc_g, acc_o, f"accumulation (mode {mode})")
        _same(out_g, out_o, f"rgba8 (mode {mode})")
        r.close()


def test_wavefront_config_rejects_out_of_range():
    r = rd.Renderer(8, 8)
    for pool, units in ((100, 0), (1 << 27, 0), (0, 1000), (0, (1 << 30) + 1)):
        with pytest.raises(WgptError) as ei:
            r.set_wavefront_config(pool, units)
        assert ei.value.code == 1
    r.set_wavefront_config(4096, 0)
    assert r.wavefront_config()[0] == 4096
    r.close()


def test_fp64_accumulation_and_3_sigma_agreement_with_oracle():
    """The FP64 Welford record holds the same samples as the FP32 running mean; a 4096-spp GPU
    estimate and an independent 256-spp oracle estimate agree within 3 sigma per pixel."""
    s = synth.small_scene(1, 256, 256, 4)
    packed = sc.pack_scene_data(s)
    sec = (112, 96, 32, 32)
    r = rd.Renderer(256, 256, seed_fn=lambda: 5)
    r.set_scene(s, packed=packed)
    r.set_accum_f64(True)
    for f0 in range(0, 4096, 1024):
        p = _params(s, packed, 256, 256, frame=f0, seed=5, section=sec[:2])
        r._check(r.L.wgpt_set_params(r.ctx, rd.ptr(p)), "params")
        r._check(r.L.wgpt_render(r.ctx, f0, 1024, *sec), "render")
    r.synchronize()
    mean, var, n = r.read_accum_f64()
    acc = r.read_accum()
    ys, xs = slice(96, 128), slice(112, 144)
    assert np.all(n[ys, xs] == 4096) and np.all(n[:96] == 0)
    np.testing.assert_allclose(mean[ys, xs], acc[ys, xs, :3], rtol=2e-3, atol=1e-5)
    po = _params(s, packed, 256, 256, seed=99, section=sec[:2])
    acc_o, _ = _oracle(packed, po, 256, 256, 0, 256, sec)
    mo = acc_o[ys, xs, :3].astype(np.float64)
    sigma = np.sqrt(var[ys, xs] / 4096.0 + var[ys, xs] / 256.0)
    inside = np.abs(mean[ys, xs] - mo) <= 3.0 * sigma + 1e-9
    frac = float(inside.mean())
    assert frac >= 0.98, f"only {frac:.4f} of pixel channels within 3 sigma"
    r.close()
