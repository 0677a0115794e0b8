"""The updateObjects fast path (tracer.js:2132-2164) on the GPU against the oracle.

After an animation step the reference re-packs the scene and writes objects, TLAS, planes,
list meshes and materials into its existing GPU buffers (queue.writeBuffer at offset 0): a
buffer keeps its length, so records beyond the new data stay visible to loops bounded by
arrayLength, and the light buffer keeps the records of the upload.  The oracle here renders
exactly that emulated buffer state, and the GPU must agree bit for bit.
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

W = H = 96
FAST = ("objects", "tlas", "planes", "meshes", "materials")


def _scene():
    s = synth.small_scene(4, W, H, 6)
    lamp = sc.Material("lamp", [1, 0.9, 0.8], 1.0, emittance=[1, 0.9, 0.7], emissionIntensity=6.0)
    a = s.add(sc.Sphere("lamp0", lamp, 1.5, 3.0, 1.0, 0.6))
    a.enableNEE = True
    b = s.add(sc.Cube("lamp1", lamp, -3.0, 2.0, -2.0, -2.2, 2.5, -1.4))
    b.enableNEE = True
    t = s.add(sc.Torus("torus", sc.Material("t", [0.7, 0.5, 0.3], 0.3, metallic=0.5), 1.0, 0.3))
    t.set_position(0.0, -1.0, 0.0)
    mesh = synth.displaced_icosphere(2, 0.1, seed=3)
    for i in range(3):
        m = s.add(sc.Model(f"blob{i}", sc.Material(f"blob{i}", [0.3 + 0.2 * i, 0.5, 0.6], 0.4), mesh))
        m.set_position(-2.0 + 2.0 * i, 0.5, 2.5)
        m.scale_set(0.7)
    lm = s.add(sc.Model("listed", sc.Material("listed", [0.8, 0.3, 0.3], 0.6), mesh, in_scene_bvh=False))
    lm.set_position(2.5, -1.5, 1.0)
    s.add(sc.Plane("back", sc.Material("back", [0.6, 0.6, 0.7], 0.9), 0, 0, 1, -6.0))
    return s


def _as_bytes(a):
    return np.ascontiguousarray(a).view(np.uint8).reshape(-1)


def _emulated(old: sc.PackedScene, new: sc.PackedScene) -> sc.PackedScene:
    """The buffers the GPU holds after the fast path: each rewritten buffer keeps its length."""
    out = sc.PackedScene(**{**old.__dict__})
    for name in FAST:
        o, n = _as_bytes(getattr(old, name)), _as_bytes(getattr(new, name))
        assert n.size <= o.size
        buf = o.copy()
        buf[:n.size] = n
        setattr(out, name, buf)
    out.total_light_power = new.total_light_power
    return out


def _params(scene, packed, frame):
    scene.camera.aspect = 1.0
    scene.camera.update_rays2()
    return sc.pack_params(scene, packed, W, H, frame, 1, (0, 0))


def _oracle(packed, params, first, reps, acc=None):
    """Oracle frames first..first+reps-1 accumulated onto `acc` (zeros by default)."""
    acc = np.zeros((H, W, 4), np.float32) if acc is None else acc.copy()
    out = np.zeros((H, W, 4), np.uint8)
    assert oracle.render(oracle.OracleScene(packed), params, first, reps, (0, 0, W, H), acc, out,
                         oracle.default_threads()) == 0
    return acc, out


def _gpu(r, params, first, reps):
    r._check(r.L.wgpt_set_params(r.ctx, rd.ptr(params)), "set_params")
    r._check(r.L.wgpt_render(r.ctx, first, reps, 0, 0, W, H), "render")
    r.synchronize()
    return r.read_accum(), r.read_output()


def _same(a, b, what):
    bad = ~((a == b) | (np.isnan(a) & np.isnan(b)))
    assert not bad.any(), f"{what}: {int(bad.sum())} values differ"


@pytest.mark.parametrize("mode", [0, 1])
def test_animation_step_fast_path_bitexact(mode):
    s = _scene()
    r = rd.Renderer(W, H)
    r.set_scene(s)
    r._check(r.L.wgpt_set_render_mode(r.ctx, mode), "mode")
    old = r.packed
    p0 = _params(s, old, 0)
    acc0, _ = _oracle(old, p0, 0, 2)
    _same(_gpu(r, p0, 0, 2)[0], acc0, "accumulation before the update")
    # one animation step, keeping the accumulation as updateObjects does: move primitives, an
    # instance, a light object and the listed mesh; recolour a material
    objs = {o.name: o for o in s.objects}
    objs["sphere0"].set_position(0.5, 1.0, -1.0)
    objs["blob1"].set_position(0.0, 1.5, 2.0)
    objs["torus"].rotate(0.6, 1, 0, 0)
    objs["lamp1"].set_position(-2.0, 2.5, -1.0)       # the light record keeps the old box
    objs["listed"].set_position(2.0, -1.0, 1.5)
    objs["blob0"].material.color = [0.9, 0.2, 0.1]
    objs["blob0"].material.roughness = 0.1
    assert r.update_objects() is True
    new = r.packed
    emu = _emulated(old, new)
    params = _params(s, new, 2)
    acc_o, out_o = _oracle(emu, params, 2, 3, acc0)
    acc_g, out_g = _gpu(r, params, 2, 3)
    _same(acc_g, acc_o, f"accumulation after update (mode {mode})")
    _same(out_g, out_o, f"rgba8 after update (mode {mode})")
    # the stale light record is what the oracle used: the fresh scene renders differently
    fresh, _ = _oracle(new, params, 2, 3, acc0)
    assert not np.array_equal(fresh, acc_o)
    r.close()


def test_removed_records_stay_in_the_buffers():
    """Dropping a plane and an object shrinks the packed data; the buffers keep their tails (the
    stale plane is still traced, as arrayLength in the reference still counts it)."""
    s = _scene()
    r = rd.Renderer(W, H)
    r.set_scene(s)
    old = r.packed
    s.objects = [o for o in s.objects if o.name not in ("back", "sphere2")]
    assert r.update_objects() is True
    new = r.packed
    assert _as_bytes(new.planes).size < _as_bytes(old.planes).size
    emu = _emulated(old, new)
    params = _params(s, new, 0)
    acc_o, out_o = _oracle(emu, params, 0, 2)
    acc_g, out_g = _gpu(r, params, 0, 2)
    _same(acc_g, acc_o, "accumulation")
    _same(out_g, out_o, "rgba8")
    r.close()


def test_growth_or_new_flags_take_the_slow_path():
    s = _scene()
    r = rd.Renderer(W, H)
    r.set_scene(s)
    s.add(sc.Sphere("extra", sc.Material("x", [0.2, 0.8, 0.2], 0.5), 0.0, 3.5, 0.0, 0.4))
    assert r.update_objects() is False           # objects no longer fit: full upload
    params = _params(s, r.packed, 0)
    acc_o, _ = _oracle(r.packed, params, 0, 2)
    acc_g, _ = _gpu(r, params, 0, 2)
    _same(acc_g, acc_o, "accumulation after the slow path")
    s.add(sc.Cylinder("cyl", sc.Material("c", [0.5, 0.5, 0.5], 0.5), 0.5))   # a new primitive kind
    packed = sc.pack_scene_data(s)
    desc = rd.scene_desc(packed)
    assert r.L.wgpt_update_objects(r.ctx, rd.C.byref(desc)) == 7
    r.close()


def test_update_rejects_bad_records_and_keeps_the_scene():
    s = _scene()
    r = rd.Renderer(W, H)
    r.set_scene(s)
    p = r.packed
    params = _params(s, p, 0)
    before, _ = _gpu(r, params, 0, 1)
    bad = sc.PackedScene(**{**p.__dict__})
    ob = _as_bytes(p.objects).copy().view(np.int32).reshape(-1, 24)
    ob[0, 16] = 10_000                              # material index out of range
    bad.objects = ob.view(np.uint8).reshape(-1)
    desc = rd.scene_desc(bad)
    assert r.L.wgpt_update_objects(r.ctx, rd.C.byref(desc)) == 2
    bad = sc.PackedScene(**{**p.__dict__})
    ob = _as_bytes(p.objects).copy().view(np.uint32).reshape(-1, 24)
    mesh_rows = np.nonzero(ob[:, 18] == 0)[0]
    ob[mesh_rows[0], 19] = 7                        # a mesh instance of a BLAS root never uploaded
    bad.objects = ob.view(np.uint8).reshape(-1)
    desc = rd.scene_desc(bad)
    assert r.L.wgpt_update_objects(r.ctx, rd.C.byref(desc)) == 7
    after, _ = _gpu(r, params, 0, 1)
    _same(after, before, "scene unchanged by rejected updates")
    with pytest.raises(WgptError):
        r._check(r.L.wgpt_update_objects(r.ctx, None), "null descriptor")
    r.close()


def test_textured_scene_update_keeps_texture_layers():
    """Materials that start or stop sampling a resident texture layer, and moved textured
    objects: the layers keep the indices of the upload (updateObjects does not prepare the
    texture array again), and a texture that was never prepared packs as -1."""
    s = synth.textured_scene(2, W, H, 5)
    r = rd.Renderer(W, H)
    r.set_scene(s)
    old = r.packed
    mats = {m.name: m for m in s.get_materials()}
    mats["rough"].albedoTex = mats["cutout"].albedoTex        # a resident layer
    mats["glow"].normalTex = sc.Texture(np.full((64, 64, 4), 128, np.uint8), "never prepared")
    mats["bumpy"].normalTex = None
    objs = {o.name: o for o in s.objects}
    objs["cut_sphere"].set_position(-1.0, 0.8, 0.5)
    assert r.update_objects() is True
    new = r.packed
    m = _as_bytes(new.materials).view(np.int32).reshape(-1, 36)
    idx = {name: i for i, name in enumerate(x.name for x in s.get_materials())}
    assert m[idx["rough"], 24] == mats["cutout"].albedoTex.texIndex >= 0
    assert m[idx["glow"], 25] == -1
    emu = _emulated(old, new)
    params = _params(s, new, 0)
    acc_o, out_o = _oracle(emu, params, 0, 3)
    acc_g, out_g = _gpu(r, params, 0, 3)
    _same(acc_g, acc_o, "accumulation")
    _same(out_g, out_o, "rgba8")
    r.close()
