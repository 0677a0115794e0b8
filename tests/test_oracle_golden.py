"""The oracle and the host packers against committed fixtures (tests/golden/golden.npz, made by
tests/golden/make_golden.py) and against independent restatements."""
from __future__ import annotations

import hashlib
from pathlib import Path

import numpy as np
import pytest

import oracle
from oracle import host_oracle as ho
from webgpuraytracer_b200 import renderer as rd
from webgpuraytracer_b200 import scene as sc
from webgpuraytracer_b200 import synth

G = np.load(Path(__file__).resolve().parent / "golden" / "golden.npz")
import importlib.util
_spec = importlib.util.spec_from_file_location("make_golden", Path(__file__).resolve().parent / "golden" / "make_golden.py")
mg = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(mg)


@pytest.mark.parametrize("k", range(len(mg.PCG_CASES)))
def test_pcg_stream_matches_plain_integer_restatement(k):
    idx, frame, seed = mg.PCG_CASES[k]
    got = oracle.rng_stream(idx, frame, seed, 64)
    np.testing.assert_array_equal(got, mg.pcg_stream(idx, frame, seed, 64))
    np.testing.assert_array_equal(got, G[f"pcg_{k}"])
    assert np.all((got >= 0) & (got <= 1))


def test_packed_small_scene_matches_fixture():
    _, _, dig = mg.small_scene_digests()
    for name, d in dig.items():
        assert d == str(G[f"sha_{name}"]), f"packed {name} changed"


def test_oracle_render_matches_fixture():
    s, p, _ = mg.small_scene_digests()
    params = G["render_params"]
    acc = np.zeros((48, 48, 4), np.float32)
    out = np.zeros((48, 48, 4), np.uint8)
    assert oracle.render(oracle.OracleScene(p), params, 0, 2, (0, 0, 48, 48), acc, out, 2) == 0
    np.testing.assert_array_equal(acc, G["render_accum"])
    np.testing.assert_array_equal(out, G["render_out"])


def test_oracle_render_thread_count_invariant():
    s, p, _ = mg.small_scene_digests()
    params = G["render_params"]
    res = []
    for threads in (1, 3):
        acc = np.zeros((48, 48, 4), np.float32)
        out = np.zeros((48, 48, 4), np.uint8)
        oracle.render(oracle.OracleScene(p), params, 0, 2, (0, 0, 48, 48), acc, out, threads)
        res.append(acc)
    np.testing.assert_array_equal(res[0], res[1])


def test_oracle_denoise_matches_fixture():
    u = rd.denoise_uniforms(40, 30, passes=3)
    f, c, o = oracle.denoise(G["dn_color"], G["dn_gbuf"], u, rd.step_schedule(3, "intended"), 2)
    np.testing.assert_array_equal(f, G["dn_filtered"])
    np.testing.assert_array_equal(o, G["dn_out"])
    assert np.all(np.isfinite(f))


def test_denoise_step_schedules():
    np.testing.assert_array_equal(rd.step_schedule(5, "intended"), [1, 2, 4, 8, 16])
    np.testing.assert_array_equal(rd.step_schedule(5, "as_run"), [16] * 5)
    np.testing.assert_array_equal(rd.step_schedule(4, "as_run"), [8] * 4)


def test_resample_identity_ratio():
    rng = np.random.default_rng(1)
    src = rng.integers(0, 256, (17, 23, 4), dtype=np.uint8)
    dst = oracle.resample(src, 23, 17, 1.0, 1.0)
    # sample positions land on texel centres minus 0.5: a half-texel shift of the bilinear filter
    assert dst.shape == (17, 23, 4) and np.all(dst[..., 3] == 255)
    same = oracle.resample(src, 23, 17, 1.0, 1.0)
    np.testing.assert_array_equal(dst, same)


MATS = [
    dict(ior=1.5, specular_tint=0.0, sheen=0.0, sheen_tint=0.5, subsurface=0.0, subsurface_tint=[1, 1, 1],
         clearcoat=0.0, clearcoat_gloss=1.0, clearcoat_ior=1.5, transmission=0.0, metallic=0.0, roughness=0.8),
    dict(ior=1.8, specular_tint=0.4, sheen=0.6, sheen_tint=0.3, subsurface=0.3, subsurface_tint=[0.9, 0.5, 0.4],
         clearcoat=0.7, clearcoat_gloss=0.6, clearcoat_ior=1.4, transmission=0.0, metallic=0.3, roughness=0.5),
    dict(ior=1.5, specular_tint=0.0, sheen=0.0, sheen_tint=0.5, subsurface=0.0, subsurface_tint=[1, 1, 1],
         clearcoat=0.0, clearcoat_gloss=1.0, clearcoat_ior=1.5, transmission=0.9, metallic=0.0, roughness=0.6),
]


@pytest.mark.parametrize("mi", range(len(MATS)))
def test_bsdf_single_precision_within_1e5_of_double(mi):
    """eval/pdf in FP32 (oracle, same arithmetic as the kernels) vs an FP64 restatement, on a
    well-conditioned domain: roughness >= 0.5, directions away from grazing (|cos| > 0.2) and
    away from the half-vector singularities."""
    m = MATS[mi]
    mat = sc.Material("m", [0.6, 0.5, 0.3], m["roughness"], metallic=m["metallic"], ior=m["ior"],
                      specularTint=m["specular_tint"], sheen=m["sheen"], sheenTint=m["sheen_tint"],
                      subsurface=m["subsurface"], subsurfaceTint=[c ** (1 / 2.2) for c in m["subsurface_tint"]],
                      clearcoat=m["clearcoat"], clearcoatGloss=m["clearcoat_gloss"], clearcoatIor=m["clearcoat_ior"],
                      transmission=m["transmission"])
    buf, _ = sc.pack_data_from_schema([mat], lambda x: x.schema(), None)
    f32 = buf.view(np.float32)
    albedo = f32[0:3].astype(np.float64)
    rng = np.random.default_rng(mi)
    vl = []
    while len(vl) < 400:
        V = rng.normal(size=3); V /= np.linalg.norm(V)
        L = rng.normal(size=3); L /= np.linalg.norm(L)
        if abs(V[2]) < 0.2 or abs(L[2]) < 0.2 or V[2] < 0:
            continue
        if m["transmission"] == 0 and L[2] < 0:
            continue
        vl.append(np.concatenate([V, L]))
    vl = np.array(vl, np.float32)
    n = [0.0, 0.0, 1.0]
    f, pdf = oracle.bsdf(buf, n, f32[4], f32[3], albedo.astype(np.float32), vl)
    mref = dict(m)
    mref["subsurface_tint"] = f32[16:19].astype(np.float64)
    for k, key in ((5, "ior"), (6, "specular_tint"), (9, "sheen"), (10, "sheen_tint"), (11, "clearcoat"),
                   (12, "clearcoat_gloss"), (13, "clearcoat_ior"), (14, "transmission"), (19, "subsurface")):
        mref[key] = float(f32[k])
    for i in range(len(vl)):
        fr, pr = ho.bsdf_f64(mref, n, albedo, float(f32[4]), float(f32[3]), vl[i, :3].astype(np.float64),
                             vl[i, 3:].astype(np.float64))
        np.testing.assert_allclose(f[i], fr, rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(pdf[i], pr, rtol=1e-5, atol=1e-6)
