"""Leaf shapes the builders rarely make, on the GPU against the oracle.

The reference's TLAS builder splits down to one object per leaf below ~1M objects, and its SAH
BLAS builder makes small leaves, so the traversal's handling of wide leaves is reached only by
scenes built for it: a TLAS set by hand (as a caller of the C ABI may) with one leaf of all 71
objects, or a leaf of 68 spheres next to a leaf of three mesh instances (the objects after an
instance wait on the stack while its BLAS is traversed), and a BLAS leaf of 80 triangles that
share one centroid, which no SAH split separates.  Both render modes must match the oracle bit
for bit.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from webgpuraytracer_b200 import renderer as rd
from webgpuraytracer_b200 import scene as sc
from webgpuraytracer_b200 import synth
from webgpuraytracer_b200._lib import MODE_MEGAKERNEL, MODE_WAVEFRONT

pytestmark = pytest.mark.gpu

W = H = 64
SPP = 4


def _same(a, b, what):
    bad = ~((a == b) | (np.isnan(a) & np.isnan(b)))
    assert not bad.any(), f"{what}: {int(bad.sum())} values differ"


def _render_both(scene, packed, mode):
    scene.camera.aspect = 1.0
    scene.camera.update_rays2()
    params = sc.pack_params(scene, packed, W, H, 0, 1, (0, 0))
    acc_o = np.zeros((H, W, 4), np.float32)
    out_o = np.zeros((H, W, 4), np.uint8)
    assert oracle.render(oracle.OracleScene(packed), params, 0, SPP, (0, 0, W, H), acc_o, out_o,
                         oracle.default_threads()) == 0
    r = rd.Renderer(W, H)
    r.set_scene(scene, packed=packed)
    r.set_render_mode(mode)
    r._check(r.L.wgpt_set_params(r.ctx, rd.ptr(params)), "set_params")
    r._check(r.L.wgpt_render(r.ctx, 0, SPP, 0, 0, W, H), "render")
    r.synchronize()
    acc_g, out_g = r.read_accum(), r.read_output()
    r.close()
    return acc_o, out_o, acc_g, out_g


def _fan_mesh(n=80, seed=5):
    """n triangles (p, q, -(p+q)) on a 1/64 grid: every centroid is exactly the origin."""
    rng = np.random.default_rng(seed)
    p = rng.integers(-48, 49, (n, 3)) / 64.0
    q = rng.integers(-48, 49, (n, 3)) / 64.0
    v = np.stack([p, q, -(p + q)], 1).reshape(-1, 3)
    e1, e2 = v[1::3] - v[0::3], v[2::3] - v[0::3]
    nrm = np.cross(e1, e2)
    nrm /= np.maximum(np.linalg.norm(nrm, axis=1, keepdims=True), 1e-12)
    normals = np.repeat(nrm, 3, 0)
    uvs = np.zeros((3 * n, 2))
    return sc.ModelData("fan", v, normals, uvs, np.arange(3 * n)).generate_bvh()


def _fan_scene():
    s = synth.small_scene(3, W, H, 4)
    mat = sc.Material("fan", [0.8, 0.6, 0.3], 0.4, metallic=0.3)
    m = s.add(sc.Model("fan", mat, _fan_mesh()))
    m.set_position(0.0, 1.0, 0.0)
    m.scale_set(2.0)
    return s


@pytest.mark.parametrize("mode", [MODE_WAVEFRONT, MODE_MEGAKERNEL])
def test_wide_blas_leaf_bitexact(mode):
    s = _fan_scene()
    p = sc.pack_scene_data(s)
    nodes = np.ascontiguousarray(p.bvh).view(np.uint32).reshape(-1, 8)
    assert nodes[:, 3].max() == 80                  # one leaf holds every triangle
    acc_o, out_o, acc_g, out_g = _render_both(s, p, mode)
    _same(acc_g, acc_o, "accumulation")
    _same(out_g, out_o, "rgba8")


def _tlas_scene():
    s = synth.small_scene(4, W, H, 4)
    s.objects = [o for o in s.objects if o.type == "Plane"]
    rng = np.random.default_rng(9)
    for i in range(68):
        mat = sc.Material(f"m{i}", list(rng.uniform(0.2, 0.9, 3)), float(rng.uniform(0.1, 1.0)),
                          metallic=float(rng.uniform(0, 1)))
        x, y, z = rng.uniform(-4, 4), rng.uniform(-0.5, 3), rng.uniform(-4, 4)
        s.add(sc.Sphere(f"s{i}", mat, x, y, z, float(rng.uniform(0.15, 0.45))))
    mesh = synth.displaced_icosphere(2, 0.1, seed=2)
    for i in range(3):
        m = s.add(sc.Model(f"blob{i}", sc.Material(f"b{i}", [0.4, 0.5 + 0.1 * i, 0.7], 0.3), mesh))
        m.set_position(-2.0 + 2.0 * i, 1.0, 1.5)
        m.scale_set(0.8)
    return s


def _node(lo, hi, num, nxt):
    rec = np.zeros(8, np.uint32)
    rec[0:3] = np.asarray(lo, np.float32).view(np.uint32)
    rec[3] = num
    rec[4:7] = np.asarray(hi, np.float32).view(np.uint32)
    rec[7] = nxt
    return rec


@pytest.mark.parametrize("mode", [MODE_WAVEFRONT, MODE_MEGAKERNEL])
@pytest.mark.parametrize("shape", ["one_leaf", "two_leaves"])
def test_hand_made_tlas_leaves_bitexact(mode, shape):
    s = _tlas_scene()
    p = sc.pack_scene_data(s)
    n = np.ascontiguousarray(p.objects).size // 96
    assert n == 71
    root = np.ascontiguousarray(p.tlas).view(np.uint32).reshape(-1, 8)[0]
    lo, hi = root[0:3].view(np.float32), root[4:7].view(np.float32)
    if shape == "one_leaf":          # all 71 objects, three mesh instances last: node form + rest
        tlas = _node(lo, hi, n, 0)[None]
    else:                            # 68 spheres (node form), then 3 meshes (inline + rest)
        tlas = np.stack([_node(lo, hi, 0, 2), _node(lo, hi, 68, 0), _node(lo, hi, 3, 68)])
    q = sc.PackedScene(**{**p.__dict__})
    q.tlas = np.ascontiguousarray(tlas).view(np.uint8).reshape(-1)
    acc_o, out_o, acc_g, out_g = _render_both(s, q, mode)
    assert np.isfinite(acc_o).all()
    _same(acc_g, acc_o, f"accumulation ({shape})")
    _same(out_g, out_o, f"rgba8 ({shape})")
