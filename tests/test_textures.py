"""Textures on the host: the sampler's semantics, the texture-array packing and the ABI checks.

The material sampler (linear filter, repeat addressing, rgba8unorm texels; tracer.js:1965-1968,
shader.wgsl:170-173) is restated in float64 numpy here and compared with the oracle's FP32 form;
the packing follows Scene.getTextures / prepareTextureArray (tracer.js:1643-1653, 1919-1953).
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from webgpuraytracer_b200 import scene as sc
from webgpuraytracer_b200 import synth


def _bilinear_repeat(tex: np.ndarray, layer: int, uv: np.ndarray) -> np.ndarray:
    img = tex[layer].astype(np.float64) / 255.0
    h, w = img.shape[:2]
    fx = uv[:, 0].astype(np.float64) * w - 0.5
    fy = uv[:, 1].astype(np.float64) * h - 0.5
    x0, y0 = np.floor(fx), np.floor(fy)
    tx, ty = (fx - x0)[:, None], (fy - y0)[:, None]
    xa, ya = np.mod(x0, w).astype(int), np.mod(y0, h).astype(int)
    xb, yb = (xa + 1) % w, (ya + 1) % h
    top = img[ya, xa] * (1 - tx) + img[ya, xb] * tx
    bot = img[yb, xa] * (1 - tx) + img[yb, xb] * tx
    return top * (1 - ty) + bot * ty


def test_sampler_matches_float64_bilinear_repeat():
    rng = np.random.default_rng(3)
    tex = rng.integers(0, 256, (3, 16, 24, 4), dtype=np.uint8)
    uv = np.concatenate([rng.uniform(-3, 3, (4000, 2)),
                         np.array([[0, 0], [1, 1], [0.5 / 24, 0.5 / 16], [-1e-7, 1 - 1e-7], [7.25, -2.5]])])
    uv = uv.astype(np.float32)
    for layer in range(3):
        got = oracle.sample_texture(tex, layer, uv)
        ref = _bilinear_repeat(tex, layer, uv)
        # FP32 texel coordinates (|uv * size| < 80) carry up to ~80 * 2^-24 of position error
        assert np.abs(got - ref).max() < 1e-5
    # texel centres return the texel exactly; a negative layer samples as vec4(1)
    centre = np.array([[(5 + 0.5) / 24, (3 + 0.5) / 16]], np.float32)
    assert np.array_equal(oracle.sample_texture(tex, 1, centre)[0], (tex[1, 3, 5] / np.float32(255)).astype(np.float32))
    assert np.array_equal(oracle.sample_texture(tex, -1, centre)[0], np.ones(4, np.float32))


def test_sampler_non_finite_coordinates_are_defined():
    tex = np.arange(2 * 2 * 4, dtype=np.uint8).reshape(1, 2, 2, 4) * 10
    uv = np.array([[np.nan, 0.25], [np.inf, 0.25], [-np.inf, 0.25], [0.0, np.nan]], np.float32)
    got = oracle.sample_texture(tex, 0, uv)
    assert np.isfinite(got).all()
    # a non-finite coordinate samples as coordinate 0 (the texel grid origin, -0.5 texel off-centre)
    assert np.array_equal(got[0], got[1]) and np.array_equal(got[1], got[2])


def test_texture_array_order_and_indices():
    t = synth.texture_set(8, 1)
    a = sc.Material("a", [1, 1, 1], 0.5, normalTex=t["normal"], albedoTex=t["albedo"])
    b = sc.Material("b", [1, 1, 1], 0.5, metallicTex=t["metallic"], albedoTex=t["albedo"], emissiveTex=t["emissive"])
    s = sc.Scene(16, 16)
    s.add(sc.Sphere("s0", a, 0, 0, 0, 1))
    s.add(sc.Sphere("s1", b, 3, 0, 0, 1))
    p = sc.pack_scene_data(s)
    # material order, then emissive, albedo, normal, height, roughness, metallic within one
    order = [t["albedo"], t["normal"], t["emissive"], t["metallic"]]
    assert [x.texIndex for x in order] == [0, 1, 2, 3]
    assert p.textures.shape == (4, 8, 8, 4)
    for i, x in enumerate(order):
        assert np.array_equal(p.textures[i], x.image)
    m = p.materials.view(np.int32).reshape(-1, 36)
    assert m[0, 23:29].tolist() == [-1, 0, 1, -1, -1, -1]
    assert m[1, 23:29].tolist() == [2, 0, -1, -1, -1, 3]
    assert not p.flags & sc.HAS_HEIGHTMAPS


def test_textures_need_a_common_size_and_height_maps_set_the_flag():
    s = sc.Scene(16, 16)
    s.add(sc.Sphere("s0", sc.Material("a", albedoTex=sc.Texture(np.zeros((4, 4, 4), np.uint8))), 0, 0, 0, 1))
    s.add(sc.Sphere("s1", sc.Material("b", albedoTex=sc.Texture(np.zeros((8, 8, 4), np.uint8))), 3, 0, 0, 1))
    with pytest.raises(ValueError):
        sc.pack_scene_data(s)
    s = sc.Scene(16, 16)
    s.add(sc.Sphere("s0", sc.Material("a", heightTex=sc.Texture(np.zeros((4, 4, 4), np.uint8))), 0, 0, 0, 1))
    assert sc.pack_scene_data(s).flags & sc.HAS_HEIGHTMAPS


def test_emissive_textured_objects_are_not_lights():
    t = synth.texture_set(8, 1)
    glow = sc.Material("g", [1, 1, 1], 1.0, emittance=[1, 1, 1], emissionIntensity=5.0, emissiveTex=t["emissive"])
    plain = sc.Material("p", [1, 1, 1], 1.0, emittance=[1, 1, 1], emissionIntensity=5.0)
    s = sc.Scene(16, 16)
    a = s.add(sc.Sphere("a", glow, 0, 0, 0, 1))
    b = s.add(sc.Sphere("b", plain, 3, 0, 0, 1))
    a.enableNEE = b.enableNEE = True
    assert sc.Scene.light_power(a)[0] == 0.0
    assert sc.Scene.light_power(b)[0] > 0.0


def test_textured_scene_oracle_effects():
    """The textured scene renders finite values that differ from the same scene with its texture
    indices cleared on most pixels (the maps are read)."""
    s = synth.textured_scene(1, 48, 48, 4, tex_size=16)
    p = sc.pack_scene_data(s)
    s.camera.update_rays2()
    params = sc.pack_params(s, p, 48, 48, 0, 1, (0, 0))
    acc = np.zeros((48, 48, 4), np.float32)
    out = np.zeros((48, 48, 4), np.uint8)
    assert oracle.render(oracle.OracleScene(p), params, 0, 2, (0, 0, 48, 48), acc, out, oracle.default_threads()) == 0
    m = p.materials.view(np.int32).reshape(-1, 36).copy()
    m[:, 23:29] = -1
    plain = sc.PackedScene(**{**p.__dict__})
    plain.materials = m.view(np.uint8).reshape(-1)
    plain.textures = None
    acc2 = np.zeros_like(acc)
    out2 = np.zeros_like(out)
    assert oracle.render(oracle.OracleScene(plain), params, 0, 2, (0, 0, 48, 48), acc2, out2,
                         oracle.default_threads()) == 0
    assert np.isfinite(acc).all() and np.isfinite(acc2).all()
    assert (np.abs(acc - acc2)[..., :3].max(-1) > 1e-3).mean() > 0.3


def test_parallax_scene_oracle():
    """Height fields shift the texture coordinates and shadow: the parallax scene renders finite
    values that differ from the same scene with HAS_HEIGHTMAPS cleared."""
    s = synth.textured_scene(1, 48, 48, 4, tex_size=16, pom=True)
    p = sc.pack_scene_data(s)
    assert p.flags & sc.HAS_HEIGHTMAPS
    s.camera.update_rays2()
    params = sc.pack_params(s, p, 48, 48, 0, 1, (0, 0))
    out = np.zeros((48, 48, 4), np.uint8)
    accs = []
    for flags in (p.flags, p.flags & ~sc.HAS_HEIGHTMAPS):
        q = sc.PackedScene(**{**p.__dict__})
        q.flags = flags
        acc = np.zeros((48, 48, 4), np.float32)
        assert oracle.render(oracle.OracleScene(q), params, 0, 2, (0, 0, 48, 48), acc, out,
                             oracle.default_threads()) == 0
        accs.append(acc)
    assert np.isfinite(accs[0]).all()
    assert (np.abs(accs[0] - accs[1])[..., :3].max(-1) > 1e-3).mean() > 0.05
