"""Opt-in alias-table environment sampling on the GPU.

The reference draws environment light samples by binary search over its CDF
(shader.wgsl:192-254); ENV_ALIAS draws the same texel distribution from an alias table in O(1).
It consumes the same random numbers and returns the same pdf, so it is checked statistically:
with the FP64 per-pixel accumulators, the two modes' means agree within their standard errors
and their per-sample variances match.  Uploading an alias table without switching to it leaves
the default path bit for bit unchanged.
"""
from __future__ import annotations

import numpy as np
import pytest

from webgpuraytracer_b200 import renderer as rd
from webgpuraytracer_b200 import synth
from webgpuraytracer_b200._lib import MODE_MEGAKERNEL, MODE_WAVEFRONT, WgptError

pytestmark = pytest.mark.gpu

W, H, SPP = 96, 64, 512


def _scene():
    s = synth.flagship_scene(1, W, H, 4, instances=8, prims=8, subdivisions=3)
    s.camera.aspect = W / H
    return s


def _run(scene, env, mode=MODE_WAVEFRONT):
    r = rd.Renderer(W, H)
    r.set_scene(scene)
    r.set_render_mode(mode)
    if env is not None:
        r.set_env_sampling(env)
    if mode == MODE_WAVEFRONT:
        r.set_accum_f64(True)
    r.render(tsize=max(W, H), reps=SPP)
    acc = r.read_accum()
    mean = var = None
    if mode == MODE_WAVEFRONT:
        mean, var, n = r.read_accum_f64()
        assert np.all(n == SPP)
    r.close()
    return mean, var, acc


def test_alias_sampling_agrees_statistically():
    s = _scene()
    m_cdf, v_cdf, acc_cdf = _run(s, None)
    m_al, v_al, acc_al = _run(s, rd.ENV_ALIAS)
    assert np.isfinite(m_al).all() and np.isfinite(v_al).all()
    assert not np.array_equal(acc_al, acc_cdf)              # the alias path did run
    se2 = (v_cdf + v_al) / SPP
    live = se2 > 1e-12
    z = (m_al - m_cdf)[live] / np.sqrt(se2[live])
    # the two modes share their random numbers, so their difference has less variance than two
    # independent estimates: only upper bounds on the spread are meaningful
    assert np.mean(z * z) < 1.5, np.mean(z * z)
    assert np.mean(np.abs(z) > 5.0) < 2e-3
    zg = (m_al - m_cdf)[live].sum() / np.sqrt(se2[live].sum())
    assert abs(zg) < 5.0, zg
    # the same sampling distribution: where the environment samples differ, the per-sample
    # variances agree (median over pixels; the mean is carried by a few heavy-tailed pixels)
    differ = np.any(m_al != m_cdf, axis=-1) & (v_cdf.mean(-1) > 1e-12)
    assert differ.sum() > 100, int(differ.sum())
    r = v_al.mean(-1)[differ] / v_cdf.mean(-1)[differ]
    ratio = np.median(r)
    assert 0.8 < ratio < 1.25, (ratio, np.quantile(r, [0.1, 0.25, 0.75, 0.9]), int(differ.sum()))


def test_alias_sampling_is_the_same_in_both_render_modes():
    s = _scene()
    _, _, wave = _run(s, rd.ENV_ALIAS, MODE_WAVEFRONT)
    _, _, mega = _run(s, rd.ENV_ALIAS, MODE_MEGAKERNEL)
    assert np.array_equal(wave, mega)


def test_uploaded_table_leaves_cdf_mode_bitexact():
    s = _scene()
    _, _, plain = _run(s, None)
    r = rd.Renderer(W, H)
    r.set_scene(s)
    r.set_env_sampling(rd.ENV_ALIAS)                        # builds and uploads the table
    r.set_env_sampling(rd.ENV_CDF)
    r.set_accum_f64(True)
    r.render(tsize=max(W, H), reps=SPP)
    assert np.array_equal(r.read_accum(), plain)
    r.close()


def test_alias_mode_needs_a_table():
    r = rd.Renderer(W, H)
    with pytest.raises(WgptError):                          # no scene yet
        r._check(r.L.wgpt_set_env_sampling(r.ctx, rd.ENV_ALIAS), "set_env_sampling")
    s = _scene()
    r.set_scene(s)
    with pytest.raises(WgptError):                          # scene without sky_alias
        r._check(r.L.wgpt_set_env_sampling(r.ctx, rd.ENV_ALIAS), "set_env_sampling")
    with pytest.raises(WgptError):
        r._check(r.L.wgpt_set_env_sampling(r.ctx, 2), "set_env_sampling")
    bad = s.background.build_env_alias()
    bad[5, 1] = bad.shape[0]                                # alias out of range
    r.packed.sky_alias = bad
    desc = rd.scene_desc(r.packed)
    assert r.L.wgpt_upload_scene(r.ctx, rd.C.byref(desc)) != 0
    r.close()
