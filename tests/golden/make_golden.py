"""Generates tests/golden/golden.npz: fixtures that pin the oracle and the host packers.

    python tests/golden/make_golden.py

Contents: PCG streams from an independent pure-Python restatement of rand_pcg
(shader.wgsl:146-154, 2280-2282); SHA-256 digests of every packed buffer of the small
configuration's scene (packers + native builders); an oracle render (48x48, 2 spp) and an
oracle denoise of a seeded synthetic input.
"""
from __future__ import annotations

import hashlib
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from webgpuraytracer_b200 import renderer as rd  # noqa: E402
from webgpuraytracer_b200 import scene as sc  # noqa: E402
from webgpuraytracer_b200 import synth  # noqa: E402

OUT = Path(__file__).resolve().parent / "golden.npz"
PCG_CASES = [(0, 0, 1), (12345, 7, 1), (65535, 15, 1), (1920 * 1080 - 1, 63, 987654321), (77, 0, 0)]


def pcg_stream(idx: int, frame: int, seed: int, n: int) -> np.ndarray:
    """PCG-RXS-M-XS 32 with the reference's seeding and discard, in plain integers."""
    m = 0xFFFFFFFF
    state = ((idx * 1973 + frame * 9277 + seed * 26699) & m) | 1
    out = []
    for k in range(n + 1):
        s = state
        state = (s * 747796405 + 2891336453) & m
        word = (((s >> ((s >> 28) + 4)) ^ s) * 277803737) & m
        word = ((word >> 22) ^ word) & m
        if k:
            out.append(np.float32(np.float32(word) * np.float32(2.3283064365386963e-10)))
    return np.array(out, dtype=np.float32)


def small_scene_digests():
    s = synth.small_scene(1, 48, 48, 4)
    p = sc.pack_scene_data(s)
    names = ["materials", "objects", "tlas", "meshes", "bvh", "triangles", "planes", "lights", "sky_cdf", "sky"]
    return s, p, {n: hashlib.sha256(np.ascontiguousarray(getattr(p, n)).tobytes()).hexdigest() for n in names}


def synthetic_denoise_input(w=40, h=30, seed=3):
    rng = np.random.default_rng(seed)
    color = np.ones((h, w, 4), np.float32)
    color[..., :3] = rng.exponential(0.5, (h, w, 3)).astype(np.float32)
    color[5, 5, :3] = np.nan                      # sanitised by the prepass
    color[7, 9, 0] = 2e5                          # > 1e4: invalid
    g = np.zeros((h, w, 12), np.float32)
    n = rng.normal(size=(h, w, 3))
    n /= np.linalg.norm(n, axis=2, keepdims=True)
    g[..., 0:3] = n
    g[:3, :, 0:3] = 0                              # sky rows
    g[..., 3] = rng.uniform(0, 1, (h, w))
    g[..., 4:7] = rng.uniform(0, 1, (h, w, 3))
    g[..., 7] = rng.uniform(0, 1, (h, w))
    g[..., 10] = rng.uniform(0, 1, (h, w))
    g[..., 11] = rng.uniform(0, 20, (h, w))
    return color, g


def main():
    data = {}
    for k, (idx, frame, seed) in enumerate(PCG_CASES):
        data[f"pcg_{k}"] = pcg_stream(idx, frame, seed, 64)
    s, p, dig = small_scene_digests()
    for name, d in dig.items():
        data[f"sha_{name}"] = np.array(d)
    s.camera.update_rays2()
    params = sc.pack_params(s, p, 48, 48, 0, 1)
    acc = np.zeros((48, 48, 4), np.float32)
    out = np.zeros((48, 48, 4), np.uint8)
    assert oracle.render(oracle.OracleScene(p), params, 0, 2, (0, 0, 48, 48), acc, out, 1) == 0
    data["render_params"] = params
    data["render_accum"] = acc
    data["render_out"] = out
    color, g = synthetic_denoise_input()
    u = rd.denoise_uniforms(40, 30, passes=3)
    f, c, o = oracle.denoise(color, g, u, rd.step_schedule(3, "intended"), 1)
    data["dn_color"], data["dn_gbuf"], data["dn_filtered"], data["dn_out"] = color, g, f, o
    np.savez_compressed(OUT, **data)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes)")


if __name__ == "__main__":
    main()
