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
    """Converged estimates of a 32 x 32 crop: the GPU with FP64 Welford accumulation at 65,536
    samples against the CPU restatement with FP64 accumulation at 16,384 samples, independent
    sample streams (seeds 5 and 99).  Per pixel channel the difference of the means is compared
    with sigma = sqrt(var_gpu / n_gpu + var_cpu / n_cpu) from each side's own sample variance.
    For Gaussian estimates 99.73 % of the 3,072 channels fall within 3 sigma (8.3 outside
    expected, standard deviation 2.9); the test allows 20 outside (0.9935), and requires the
    mean squared z-score to be near 1 (0.8 .. 1.25), which a biased or mis-scaled estimator
    fails.  The FP64 record also holds exactly the samples of the FP32 running mean."""
    s = synth.small_scene(1, 256, 256, 4)
    packed = sc.pack_scene_data(s)
    sec = (112, 96, 32, 32)
    n_gpu, n_cpu = 65536, 16384
    r = rd.Renderer(256, 256, seed_fn=lambda: 5)
    r.set_scene(s, packed=packed)
    r.set_accum_f64(True)
    for f0 in range(0, n_gpu, 8192):
        p = _params(s, packed, 256, 256, frame=f0, seed=5, section=sec[:2])
        r._check(r.L.wgpt_set_params(r.ctx, rd.ptr(p)), "params")
        r._check(r.L.wgpt_render(r.ctx, f0, 8192, *sec), "render")
    r.synchronize()
    mean, var, n = r.read_accum_f64()
    acc = r.read_accum()
    r.close()
    ys, xs = slice(96, 128), slice(112, 144)
    assert np.all(n[ys, xs] == n_gpu) and np.all(n[:96] == 0)
    np.testing.assert_allclose(mean[ys, xs], acc[ys, xs, :3], rtol=2e-3, atol=1e-5)
    po = _params(s, packed, 256, 256, seed=99, section=sec[:2])
    acc8 = np.zeros((256, 256, 8), np.float64)
    assert oracle.render_f64(oracle.OracleScene(packed), po, 0, n_cpu, sec, acc8) == 0
    assert np.all(acc8[ys, xs, 6] == n_cpu)
    mo = acc8[ys, xs, 0:3]
    vo = acc8[ys, xs, 3:6] / (n_cpu - 1)
    sigma = np.sqrt(var[ys, xs] / n_gpu + vo / n_cpu)
    diff = mean[ys, xs] - mo
    inside = np.abs(diff) <= 3.0 * sigma + 1e-12
    frac = float(inside.mean())
    live = sigma > 0
    z2 = float(np.mean((diff[live] / sigma[live]) ** 2))
    assert frac >= 0.9935, f"only {frac:.4f} of pixel channels within 3 sigma"
    assert 0.8 <= z2 <= 1.25, f"mean squared z-score {z2:.3f}"


@pytest.mark.parametrize("tuning", [
    {"trav_shape": 1, "shade_block": 512, "refill_closest": 24, "refill_shadow": 8, "shadow_wide": 1},
    {"trav_shape": 2, "shade_block": 256, "refill_closest": 8, "refill_shadow": 16, "shadow_wide": 0},
    {"trav_shape": 0, "shade_block": 256, "refill_closest": 32, "refill_shadow": 1, "shadow_wide": 1},
    {"trav_shape": 0, "shade_block": 512, "refill_closest": 24, "refill_shadow": 8, "shadow_wide": 0},
])
def test_kernel_variants_leave_images_unchanged(tuning):
    """Every tuned kernel variant (traversal block shape, shading block, refill thresholds, the
    4-wide or 2-wide shadow walk) renders the flagship-family crop bit for bit like the default
    variants."""
    s = synth.flagship_scene(1, 160, 120, 8)
    packed = sc.pack_scene_data(s)
    out = []
    for t in (None, tuning):
        r = rd.Renderer(160, 120, seed_fn=lambda: 3)
        r.set_scene(s, packed=packed)
        if t is not None:
            r.set_wavefront_tuning(**t)
            assert r.wavefront_tuning() == t
        r.render(tsize=160, reps=4)
        out.append((r.read_accum(), r.read_output()))
        r.close()
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1], out[1][1])


def test_wavefront_tuning_rejects_out_of_range():
    r = rd.Renderer(8, 8)
    for bad in ({"trav_shape": 3}, {"shade_block": 384}, {"refill_closest": 0}, {"refill_shadow": 33},
                {"shadow_wide": 2}):
        t = {"trav_shape": 0, "shade_block": 512, "refill_closest": 24, "refill_shadow": 8, "shadow_wide": 1}
        t.update(bad)
        with pytest.raises(WgptError) as ei:
            r.set_wavefront_tuning(**t)
        assert ei.value.code == 1
    r.close()
