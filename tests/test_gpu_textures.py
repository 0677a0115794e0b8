"""Textured materials on the GPU against the oracle, bit for bit.

The scene covers every primitive kind with albedo (alpha cut-out), normal, roughness, metallic
and emissive maps; shadow rays of the sphere and box lights and of the sky cross alpha-textured
occluders (transmittance products), and mesh and torus hits with normal maps use the tangent
frame of the last plane, sphere or cube accepted before them on the ray, as the reference does.
With height fields, main's parallax occlusion mapping (coordinate shift, the height field's
shadow test in next-event estimation and the second BSDF sample after a self-shadowed
direction) is exercised too.  Both forms of main (wavefront and single kernel) and gbuf_main
are compared.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from webgpuraytracer_b200 import renderer as rd
from webgpuraytracer_b200 import scene as sc
from webgpuraytracer_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=[(True, False), (False, False), (True, True)], ids=["sky", "plain", "pom"])
def textured(request):
    sky, pom = request.param
    s = synth.textured_scene(1, 128, 128, 6, sky=sky, pom=pom)
    p = sc.pack_scene_data(s)
    assert bool(p.flags & sc.HAS_HEIGHTMAPS) == pom
    return s, p


def _params(scene, packed, w, h):
    scene.camera.aspect = w / h
    scene.camera.update_rays2()
    return sc.pack_params(scene, packed, w, h, 0, 1, (0, 0))


def _assert_same(a, b, what):
    bad = ~((a == b) | (np.isnan(a) & np.isnan(b)))
    n = int(bad.sum())
    assert n == 0, f"{what}: {n} of {a.size} values differ; first at {np.argwhere(bad)[:5].tolist()}"


@pytest.mark.parametrize("mode", [0, 1])
def test_textured_render_bitexact(textured, mode):
    scene, packed = textured
    w = h = 128
    params = _params(scene, packed, w, h)
    acc_o = np.zeros((h, w, 4), np.float32)
    out_o = np.zeros((h, w, 4), np.uint8)
    assert oracle.render(oracle.OracleScene(packed), params, 3, 6, (0, 0, w, h), acc_o, out_o,
                         oracle.default_threads()) == 0
    r = rd.Renderer(w, h)
    r.set_scene(scene, packed=packed)
    r._check(r.L.wgpt_set_render_mode(r.ctx, mode), "mode")
    r._check(r.L.wgpt_set_params(r.ctx, rd.ptr(params)), "set_params")
    r._check(r.L.wgpt_render(r.ctx, 3, 6, 0, 0, w, h), "render")
    r.synchronize()
    _assert_same(r.read_accum(), acc_o, f"accumulation (mode {mode})")
    _assert_same(r.read_output(), out_o, f"rgba8 (mode {mode})")
    r.close()


def test_textured_gbuffer_bitexact(textured):
    scene, packed = textured
    w = h = 128
    params = _params(scene, packed, w, h)
    g_o = np.zeros((h, w, 12), np.float32)
    img_o = np.zeros((h, w, 4), np.uint8)
    assert oracle.gbuffer(oracle.OracleScene(packed), params, (0, 0, w, h), g_o, img_o, oracle.default_threads()) == 0
    r = rd.Renderer(w, h)
    r.set_scene(scene, isgbuf=True, packed=packed)
    r._check(r.L.wgpt_set_params(r.ctx, rd.ptr(params)), "set_params")
    r._check(r.L.wgpt_render_gbuffer(r.ctx, 0, 0, w, h), "gbuffer")
    r.synchronize()
    _assert_same(r.read_gbuffer(), g_o, "gbuffer")
    _assert_same(r.read_output(), img_o, "gbuffer debug image")
    r.close()


def test_textures_change_the_image(textured):
    """The device path reads the maps: clearing every texture index changes most pixels."""
    scene, packed = textured
    w = h = 64
    params = _params(scene, packed, w, h)
    r = rd.Renderer(w, h)
    r.set_scene(scene, packed=packed)
    r._check(r.L.wgpt_set_params(r.ctx, rd.ptr(params)), "set_params")
    r._check(r.L.wgpt_render(r.ctx, 0, 2, 0, 0, w, h), "render")
    r.synchronize()
    a = r.read_accum()
    m = packed.materials.view(np.int32).reshape(-1, 36).copy()
    m[:, 23:29] = -1
    plain = sc.PackedScene(**{**packed.__dict__})
    plain.materials = m.view(np.uint8).reshape(-1)
    plain.textures = None
    r2 = rd.Renderer(w, h)
    r2.set_scene(scene, packed=plain)
    r2._check(r2.L.wgpt_set_params(r2.ctx, rd.ptr(params)), "set_params")
    r2._check(r2.L.wgpt_render(r2.ctx, 0, 2, 0, 0, w, h), "render")
    r2.synchronize()
    b = r2.read_accum()
    assert np.isfinite(a).all()
    assert (np.abs(a - b)[..., :3].max(-1) > 1e-3).mean() > 0.3
    r.close()
    r2.close()
