"""Batched views: many cameras of one scene, of uneven size and sample count, traced by one path
pool in one call, give each view exactly the image a render of that view alone gives."""
from __future__ import annotations

import numpy as np
import pytest

from webgpuraytracer_b200 import renderer as rd
from webgpuraytracer_b200 import scene as sc
from webgpuraytracer_b200 import synth
from webgpuraytracer_b200._lib import WgptError

pytestmark = pytest.mark.gpu

VIEWS = [
    {"width": 96, "height": 64, "spp": 3, "eye": (18.0, 6.0, 4.0), "target": (0.0, 2.0, 0.0)},
    {"width": 48, "height": 48, "spp": 1, "eye": (-12.0, 9.0, 14.0), "target": (1.0, 1.0, -1.0)},
    {"width": 128, "height": 40, "spp": 5, "eye": (0.0, 3.0, -22.0), "target": (-2.0, 2.5, 0.0)},
    {"width": 33, "height": 71, "spp": 2, "eye": (5.0, 12.0, 20.0), "target": (0.0, 0.0, 0.0)},
]
FIRST = [0, 4, 9, 1]


@pytest.fixture(scope="module")
def flagship():
    s = synth.flagship_scene(1, 1920, 1080, 8)
    return s, sc.pack_scene_data(s)


def _same(a, b, what):
    bad = ~((a == b) | (np.isnan(a) & np.isnan(b)))
    assert int(bad.sum()) == 0, f"{what}: {int(bad.sum())} values differ"


def test_batch_equals_single_view_renders(flagship):
    scene, packed = flagship
    params = [synth.view_params(scene, packed, v, f, seed=3) for v, f in zip(VIEWS, FIRST)]
    b = rd.Renderer(16, 16)
    b.set_scene(scene, packed=packed)
    b.set_wavefront_config(2048, 0)     # fewer slots than units: views share and refill the pool
    b.set_views([(v["width"], v["height"]) for v in VIEWS])
    done = b.render_views(params, FIRST, [v["spp"] for v in VIEWS])
    assert np.all(done >= 0.0), done
    for i, (v, p) in enumerate(zip(VIEWS, params)):
        r = rd.Renderer(v["width"], v["height"])
        r.set_scene(scene, packed=packed)
        r._check(r.L.wgpt_set_params(r.ctx, rd.ptr(p)), "params")
        r._check(r.L.wgpt_render(r.ctx, FIRST[i], v["spp"], 0, 0, v["width"], v["height"]), "render")
        r.synchronize()
        acc_b, out_b = b.read_view(i)
        _same(acc_b, r.read_accum(), f"view {i} accumulation")
        _same(out_b, r.read_output(), f"view {i} rgba8")
        r.close()
    # a second call continues each view's progressive accumulation
    params2 = [synth.view_params(scene, packed, v, f + v["spp"], seed=3) for v, f in zip(VIEWS, FIRST)]
    b.render_views(params2, [f + v["spp"] for v, f in zip(VIEWS, FIRST)], [1] * len(VIEWS), timing=False)
    v = VIEWS[0]
    r = rd.Renderer(v["width"], v["height"])
    r.set_scene(scene, packed=packed)
    for p, f, n in ((params[0], FIRST[0], v["spp"]), (params2[0], FIRST[0] + v["spp"], 1)):
        r._check(r.L.wgpt_set_params(r.ctx, rd.ptr(p)), "params")
        r._check(r.L.wgpt_render(r.ctx, f, n, 0, 0, v["width"], v["height"]), "render")
    r.synchronize()
    _same(b.read_view(0)[0], r.read_accum(), "view 0 after a second call")
    r.close()
    b.close()


def test_batch_rejects_inconsistent_views(flagship):
    scene, packed = flagship
    b = rd.Renderer(16, 16)
    b.set_scene(scene, packed=packed)
    b.set_views([(32, 32), (16, 8)])
    good = [synth.view_params(scene, packed, {"width": 32, "height": 32, "eye": (0, 5, 20), "target": (0, 0, 0)}),
            synth.view_params(scene, packed, {"width": 16, "height": 8, "eye": (0, 5, 20), "target": (0, 0, 0)})]
    wrong_size = [good[0], good[0]]
    with pytest.raises(WgptError) as ei:
        b.render_views(wrong_size, [0, 0], [1, 1])
    assert ei.value.code == 1
    sky = good[1].copy()
    sky.view(np.uint32)[21] += 1            # sky_height of view 1
    with pytest.raises(WgptError) as ei:
        b.render_views([good[0], sky], [0, 0], [1, 1])
    assert ei.value.code == 1
    done = b.render_views(good, [0, 0], [0, 2])
    assert done[0] == -1.0 and done[1] >= 0.0
    b.close()


def test_views_gbuffer_and_learned_denoiser_per_view(flagship):
    """Each batched view gets its G-buffer and is finished by the learned denoiser exactly as a
    single-view renderer holding the same accumulation and G-buffer would be."""
    from webgpuraytracer_b200 import kpcn
    scene, packed = flagship
    views = VIEWS[:2]
    params = [synth.view_params(scene, packed, v, 0, seed=3) for v in views]
    b = rd.Renderer(16, 16)
    b.set_scene(scene, packed=packed)
    b.set_views([(v["width"], v["height"]) for v in views])
    b.render_views_gbuffer(params)
    b.render_views(params, [0, 0], [v["spp"] for v in views], timing=False)
    net = kpcn.Kpcn(0, seed=2)
    for i, v in enumerate(views):
        lin_b = net.denoise_view(b, i, want_linear=True)
        _, out_b = b.read_view(i)
        r = rd.Renderer(v["width"], v["height"])
        r.set_scene(scene, isgbuf=True, packed=packed)
        r._check(r.L.wgpt_set_params(r.ctx, rd.ptr(params[i])), "params")
        r._check(r.L.wgpt_render_gbuffer(r.ctx, 0, 0, v["width"], v["height"]), "gbuffer")
        r._check(r.L.wgpt_render(r.ctx, 0, v["spp"], 0, 0, v["width"], v["height"]), "render")
        r.synchronize()
        lin_r = net.denoise(r)
        _same(lin_b, lin_r, f"view {i} denoised")
        _same(out_b, r.read_output(), f"view {i} denoised rgba8")
        r.close()
    net.close()
    b.close()
