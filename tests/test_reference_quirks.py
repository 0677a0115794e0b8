"""Known answers for the reference's quirks, derived from the WGSL / JavaScript text alone.

The oracle restates shader.wgsl line by line, and the GPU kernels agree with it bit for bit; a
misreading shared by both would pass those comparisons.  Each test here computes the expected
value independently, in float64 (or exact integers) from the cited reference lines, without
calling the oracle's or the library's arithmetic, and then checks the oracle (CPU tests) and the
device (tests marked gpu) against it:

* rand_pcg's f32(word) rounding a word of 2^32 - 128 or more to exactly 1.0 (shader.wgsl:146-154);
* binary_search_cdf returning max(1, low) - 1, so a target equal to a CDF entry, at or below the
  first entry and at 1.0 picks the texel the search's `<` implies (shader.wgsl:192-206, 231-254);
* the torus normal taken through mat3(inv_matrix) without the transpose the other primitives
  use (shader.wgsl:680-681 against 669, 638);
* list meshes packed at 96 bytes (Model.getSchema, tracer.js:1406-1417) and read as 80-byte
  MeshInstance records (shader.wgsl:94-100), so a list mesh reads the zero pad as its node offset
  and its node offset as its triangle offset;
* anisotropy tilting only the sampling normal of the specular lobe (shader.wgsl:2108-2116); eval
  and pdf never read it (1831-2047);
* stale tangent frames: triangles never write SurfaceHit.tangent/bitangent, so a normal map on a
  triangle uses the frame of a plane accepted earlier on the same ray (shader.wgsl:540-541 write
  no frame; trace_plane 642-656 does).
"""
from __future__ import annotations

import math
import struct

import numpy as np
import pytest

import oracle
from webgpuraytracer_b200 import scene as sc
from webgpuraytracer_b200 import synth

M32 = 0xFFFFFFFF
PCG_A, PCG_C, PCG_OUT = 747796405, 2891336453, 277803737


# ----------------------------------------------------------------------------- PCG rounding
def pcg_word(state: int) -> int:
    """The output word of rand_pcg for `state` (shader.wgsl:149-151), in exact integers."""
    word = (((state >> ((state >> 28) + 4)) ^ state) * PCG_OUT) & M32
    return ((word >> 22) ^ word) & M32


def _round_nearest_even_f32(word: int) -> float:
    """f32(word) for a word of 2^24 or more: round to nearest, ties to even, in exact integers."""
    e = word.bit_length() - 24            # bits below the 24-bit significand
    q, r = divmod(word, 1 << e)
    half = 1 << (e - 1)
    if r > half or (r == half and q & 1):
        q += 1
    return float(q << e)


def state_for_word(word: int) -> int:
    """The state whose rand_pcg output word is `word` (the output permutation inverted)."""
    w = word
    w = w ^ (w >> 22)                     # (x >> 22) ^ x is its own inverse for shifts >= 16
    x = (w * pow(PCG_OUT, -1, 1 << 32)) & M32
    r = (x >> 28) + 4                     # the shift reads the top 4 bits, which the xor keeps
    s = x
    for _ in range(8):
        s = x ^ (s >> r)
    assert pcg_word(s) == word
    return s


def seed_reaching_one():
    """(seed, k): with pixel index 0 and sample 0, the k-th returned draw (1-based, after the
    seeding discard of shader.wgsl:2282) has output word 2^32 - 1, so rand_pcg returns 1.0."""
    target = state_for_word(M32)
    k = 1 if target % 2 == 0 else 2       # states alternate parity after the odd seed state
    s = target
    a_inv = pow(PCG_A, -1, 1 << 32)
    for _ in range(k):
        s = ((s - PCG_C) * a_inv) & M32
    assert s & 1
    seed = (s * pow(26699, -1, 1 << 32)) & M32   # rng_state = (idx*1973 + frame*9277 + seed*26699) | 1
    return seed, k


def test_pcg_rounds_the_largest_words_to_one():
    assert _round_nearest_even_f32(M32) == 2.0 ** 32
    assert _round_nearest_even_f32(M32 - 127) == 2.0 ** 32          # 2^32 - 128 rounds up (tie to even)
    assert _round_nearest_even_f32(M32 - 128) == 2.0 ** 32 - 256
    seed, k = seed_reaching_one()
    draws = oracle.rng_stream(0, 0, seed, 3)
    assert draws[k - 1] == np.float32(1.0)
    # the same stream in exact integers from the WGSL text
    s = (seed * 26699) & M32 | 1
    ref = []
    for _ in range(4):
        ref.append(np.float32(_round_nearest_even_f32(pcg_word(s))) * np.float32(2.3283064365386963e-10))
        s = (s * PCG_A + PCG_C) & M32
    np.testing.assert_array_equal(draws, np.array(ref[1:], np.float32))


@pytest.mark.gpu
def test_device_pcg_rounds_the_largest_words_to_one():
    from webgpuraytracer_b200._lib import lib, ptr
    seed, k = seed_reaching_one()
    out = np.zeros(3, np.float32)
    assert lib().wgpt_rng_stream(0, 0, 0, seed, 3, ptr(out)) == 0
    assert out[k - 1] == np.float32(1.0)
    np.testing.assert_array_equal(out, oracle.rng_stream(0, 0, seed, 3))


# ----------------------------------------------------------------------------- CDF search
SKY_W, SKY_H = 4, 2
MARGINAL = [0.0, 0.25, 1.0]                                    # sky_height + 1 entries
ROWS = [[0.0, 0.1, 0.2, 0.7, 1.0], [0.0, 0.5, 0.5, 0.75, 1.0]]  # sky_width + 1 entries each
# (u.x, u.y) -> texel (x, y) by the WGSL search: low = number of the first `size` entries below
# the target, result max(1, low) - 1 (the search never looks at the last entry of a row)
CDF_CASES = [
    ((0.0, 0.0), (0, 0)),         # at the first entry: low 0 -> 0
    ((0.1, 0.25), (0, 0)),        # equal to an entry: `<` fails on it, low 1 -> 0
    ((0.15, 0.2), (1, 0)),
    ((0.2000001, 0.0), (2, 0)),
    ((0.7, 0.0), (2, 0)),
    ((0.71, 0.0), (3, 0)),        # above every searched entry: low = size -> size - 1
    ((0.7, 0.3), (2, 1)),         # row 1: texel 1 has zero width and is never picked
    ((0.5, 0.9), (0, 1)),
    ((0.75, 0.26), (2, 1)),
    ((1.0, 1.0), (3, 1)),         # rand_pcg can return exactly 1.0
]


def cdf_scene():
    """The small configuration's objects under a 4 x 2 importance-sampled sky whose CDF is
    replaced by the hand-made one above (the search reads whatever buffer it is given)."""
    s = synth.small_scene(1, 16, 16, 2)
    texels = np.zeros((SKY_H, SKY_W, 4), np.float16)
    for y in range(SKY_H):
        for x in range(SKY_W):
            texels[y, x] = (0.5 + x, 1.0 + 0.25 * y, 2.0 - 0.5 * x, 1.0)
    s.background = sc.HDRTexture(rgba16f=texels.view(np.uint16).reshape(-1), width=SKY_W, height=SKY_H)
    packed = sc.pack_scene_data(s)
    assert packed.flags & sc.MIS_SKYBOX
    packed.sky_cdf = np.array(MARGINAL + ROWS[0] + ROWS[1], np.float32)
    packed.sky_cdf_index = SKY_H + 1
    packed.sky_total_lum = 10.0
    s.camera.update_rays2()
    params = sc.pack_params(s, packed, 16, 16, 0, 1)
    return s, packed, params, texels.astype(np.float64)


def expected_pdf(texels, x, y):
    """get_sky_pdf at the texel's centre (shader.wgsl:208-229): luminance x W x H / (total 2 pi^2)."""
    r, g, b = texels[y, x, :3]
    lum = 0.2126 * r + 0.7152 * g + 0.0722 * b
    return lum * SKY_W * SKY_H / (10.0 * 2.0 * math.pi ** 2)


def test_cdf_search_known_answers_oracle():
    _, packed, params, texels = cdf_scene()
    u2 = np.array([c[0] for c in CDF_CASES], np.float32)
    texel, pdf = oracle.sample_env(oracle.OracleScene(packed), params, u2)
    assert [tuple(int(v) for v in t) for t in texel] == [c[1] for c in CDF_CASES]
    exp = [expected_pdf(texels, x, y) for _, (x, y) in CDF_CASES]
    np.testing.assert_allclose(pdf, exp, rtol=1e-5)


@pytest.mark.gpu
def test_cdf_search_known_answers_device():
    from webgpuraytracer_b200 import renderer as rd
    from webgpuraytracer_b200._lib import ptr
    s, packed, params, texels = cdf_scene()
    r = rd.Renderer(16, 16)
    r.set_scene(s, packed=packed)
    r._check(r.L.wgpt_set_params(r.ctx, ptr(params)), "set_params")
    u2 = np.array([c[0] for c in CDF_CASES], np.float32)
    texel = np.zeros((len(u2), 2), np.uint32)
    pdf = np.zeros(len(u2), np.float32)
    r._check(r.L.wgpt_sample_env(r.ctx, ptr(u2), len(u2), ptr(texel), ptr(pdf)), "sample_env")
    r.close()
    assert [tuple(int(v) for v in t) for t in texel] == [c[1] for c in CDF_CASES]
    np.testing.assert_allclose(pdf, [expected_pdf(texels, x, y) for _, (x, y) in CDF_CASES], rtol=1e-5)


# ----------------------------------------------------------------------------- torus normal
def torus_scene():
    mat = sc.Material("m", [0.5, 0.5, 0.5], 0.5)
    s = sc.Scene(16, 16)
    t = sc.Torus("torus", mat, 1.0, 0.35)
    t.scale_set(1.6, 0.5, 0.9)            # non-uniform: mat3(inv) and its transpose differ
    t.rotate(0.6, 0.3, 1.0, 0.2)
    t.set_position(0.2, -0.1, 0.3)
    s.add(t)
    s.background = sc.HDRTexture([1.0, 1.0, 1.0])
    packed = sc.pack_scene_data(s)
    inv = np.frombuffer(packed.objects[:64].tobytes(), np.float32).astype(np.float64)
    inner = struct.unpack_from("<f", packed.objects.tobytes(), 76)[0]
    return s, packed, inv, inner


def torus_rays(inv):
    """Rays from outside aimed at points on the tube's outer equator (world space)."""
    M = np.linalg.inv(inv.reshape(4, 4).T)          # object -> world (column-major storage)
    rays = []
    for k in range(8):
        a = 2 * math.pi * (k + 0.3) / 8
        target = M @ np.array([math.cos(a) * 1.2, 0.05, math.sin(a) * 1.2, 1.0])
        origin = np.array([3.0 * math.cos(a + 0.4), 2.5, 3.0 * math.sin(a + 0.4) + 4.0])
        d = target[:3] - origin
        rays.append(np.concatenate([origin, d / np.linalg.norm(d)]))
    return np.array(rays)


def torus_expected(inv, inner, ray):
    """trace_torus (shader.wgsl:663-692) in float64: world t and the quirk normal
    normalize(mat3(inv) * local_n), plus the transposed (correct) normal for contrast."""
    Inv = inv.reshape(4, 4).T                       # Inv @ v applies inv_matrix
    lo = (Inv @ np.append(ray[:3], 1.0))[:3]
    ld = (Inv @ np.append(ray[3:], 0.0))[:3]
    scale = np.linalg.norm(ld)
    ld = ld / scale
    # (|p|^2 + R^2 - r^2)^2 = 4 R^2 (x^2 + z^2), R = 1, r = inner: a quartic in t
    R, r = 1.0, inner
    a = np.dot(ld, ld)
    b = 2 * np.dot(lo, ld)
    c = np.dot(lo, lo) + R * R - r * r
    q = np.polynomial.polynomial
    lhs = q.polymul([c, b, a], [c, b, a])
    rhs = 4 * R * R * np.array([lo[0] ** 2 + lo[2] ** 2, 2 * (lo[0] * ld[0] + lo[2] * ld[2]), ld[0] ** 2 + ld[2] ** 2])
    roots = q.polyroots(q.polysub(lhs, rhs))
    ts = sorted(x.real for x in roots if abs(x.imag) < 1e-9 and x.real > 1e-4)
    t = ts[0]
    p = lo + ld * t
    ring = np.array([p[0], 0.0, p[2]]) / math.hypot(p[0], p[2])
    ln = (p - ring) / np.linalg.norm(p - ring)
    m3 = Inv[:3, :3]                                # columns inv_matrix[0..2].xyz
    quirk = m3 @ ln
    correct = m3.T @ ln
    return t / scale, quirk / np.linalg.norm(quirk), correct / np.linalg.norm(correct)


def _check_torus(o_idx, t, nrm, rays, inv, inner):
    for i, ray in enumerate(rays):
        wt, quirk, correct = torus_expected(inv, inner, ray)
        assert o_idx[i] == 0
        assert abs(t[i] - wt) <= 1e-3 * wt
        np.testing.assert_allclose(nrm[i], quirk, atol=2e-3)
        assert np.linalg.norm(quirk - correct) > 0.05      # the case actually tells them apart


def test_torus_normal_without_transpose_oracle():
    _, packed, inv, inner = torus_scene()
    rays = torus_rays(inv)
    o, m, pr, t, nrm = oracle.trace_closest(oracle.OracleScene(packed), rays)
    _check_torus(o, t, nrm, rays, inv, inner)


@pytest.mark.gpu
def test_torus_normal_without_transpose_device():
    from webgpuraytracer_b200 import renderer as rd
    s, packed, inv, inner = torus_scene()
    r = rd.Renderer(16, 16)
    r.set_scene(s, packed=packed)
    rays = torus_rays(inv)
    o, m, pr, t, nrm = r.trace_rays(rays)
    r.close()
    _check_torus(o, t, nrm, rays, inv, inner)


# ----------------------------------------------------------------------------- list-mesh stride
def _model(name, tris):
    pos = np.array([v for tri in tris for v in tri], np.float32)
    n = len(tris)
    nrm = np.tile(np.array([0.0, 0.0, 1.0], np.float32), (3 * n, 1))
    uv = np.zeros((3 * n, 2), np.float32)
    return sc.ModelData(name, pos, nrm, uv, np.arange(3 * n)).generate_bvh()


def list_mesh_scene():
    """A mesh in the TLAS (one triangle: one BLAS node, offsets 0/0), then a list mesh of two
    triangles (packed at node offset 1, triangle offset 1).  Read at the 80-byte stride, the list
    mesh's record gives node_offset = the zero at byte 72 and tri_offset = its node offset (1) at
    byte 76: traversal walks the first mesh's single leaf (its box in the list mesh's local
    frame, one triangle, first index 0) and tests triangle 0 + 1 = the list mesh's first
    flattened triangle only."""
    m0 = _model("big", [[(-10.0, -10.0, -1.0), (10.0, -10.0, 1.0), (0.0, 10.0, 0.0)]])
    m1 = _model("pair", [[(-2.0, -1.0, 0.0), (-0.5, -1.0, 0.0), (-1.25, 1.0, 0.0)],
                         [(0.5, -1.0, 0.0), (2.0, -1.0, 0.0), (1.25, 1.0, 0.0)]])
    s = sc.Scene(16, 16)
    far = sc.Model("far", sc.Material("a", [0.5, 0.5, 0.5], 0.5), m0)
    far.set_position(0.0, 500.0, 0.0)
    s.add(far)
    s.add(sc.Model("listed", sc.Material("b", [0.5, 0.5, 0.5], 0.5), m1, in_scene_bvh=False))
    s.background = sc.HDRTexture([1.0, 1.0, 1.0])
    packed = sc.pack_scene_data(s)
    rec = packed.meshes.tobytes()
    assert len(rec) == 96                                          # one record at Model.getSchema's stride
    assert struct.unpack_from("<I", rec, 76)[0] == 1 and struct.unpack_from("<i", rec, 72)[0] == 0
    flat = np.frombuffer(packed.triangles.tobytes(), np.float32).reshape(-1, 32)
    first = flat[1, [0, 1, 2, 4, 5, 6, 8, 9, 10]].reshape(3, 3).astype(np.float64)   # list mesh flat tri 0
    second = flat[2, [0, 1, 2, 4, 5, 6, 8, 9, 10]].reshape(3, 3).astype(np.float64)
    return s, packed, first, second


def test_list_mesh_read_at_80_bytes_oracle():
    _, packed, first, second = list_mesh_scene()
    rays = []
    for tri in (first, second):
        c = tri.mean(axis=0)
        rays.append([c[0], c[1], 10.0, 0.0, 0.0, -1.0])
    o, m, pr, t, nrm = oracle.trace_closest(oracle.OracleScene(packed), np.array(rays))
    # through the list mesh's first flattened triangle: hit at z = 0, t = 10, object -1
    assert (o[0], m[0], pr[0]) == (-1, 1, 1) and abs(t[0] - 10.0) < 1e-5
    # through its second triangle: never tested at the 80-byte read, so the ray misses
    assert m[1] == -1


@pytest.mark.gpu
def test_list_mesh_read_at_80_bytes_device():
    from webgpuraytracer_b200 import renderer as rd
    s, packed, first, second = list_mesh_scene()
    r = rd.Renderer(16, 16)
    r.set_scene(s, packed=packed)
    rays = np.array([[*tri.mean(axis=0)[:2], 10.0, 0.0, 0.0, -1.0] for tri in (first, second)])
    o, m, pr, t, nrm = r.trace_rays(rays)
    r.close()
    assert (o[0], m[0], pr[0]) == (-1, 1, 1) and abs(t[0] - 10.0) < 1e-5
    assert m[1] == -1


# ----------------------------------------------------------------------------- anisotropy
def _material_bytes(**kw):
    m = sc.Material("aniso", [1.0, 1.0, 1.0], 0.0, metallic=1.0, **kw)
    m._index = 0
    buf, _ = sc.pack_data_from_schema([m], lambda x: x.schema(), sc._MAT_EMPTY)
    return np.ascontiguousarray(buf[:144])


def test_anisotropy_leaves_eval_and_pdf_alone():
    rng = np.random.default_rng(3)
    vl = rng.normal(size=(256, 6))
    vl[:, :3] /= np.linalg.norm(vl[:, :3], axis=1, keepdims=True)
    vl[:, 3:] /= np.linalg.norm(vl[:, 3:], axis=1, keepdims=True)
    vl[:, 2] = np.abs(vl[:, 2])
    vl[:, 5] = np.abs(vl[:, 5])
    n = (0.0, 0.0, 1.0)
    base = _material_bytes()
    tilted = _material_bytes(anisotropic=0.8, anisotropicRotation=0.3)
    f0, p0 = oracle.bsdf(base, n, 0.4, 1.0, (0.8, 0.7, 0.6), vl)
    f1, p1 = oracle.bsdf(tilted, n, 0.4, 1.0, (0.8, 0.7, 0.6), vl)
    np.testing.assert_array_equal(f0, f1)
    np.testing.assert_array_equal(p0, p1)


def test_anisotropy_tilts_the_sampling_normal():
    """A white metal (specular lobe probability 1) at roughness 0 (alpha = 1e-4 after the clamp):
    the VNDF half vector is the lobe's normal to within ~1e-4, so the sampled direction is the
    mirror direction about N_spec = normalize(mix(n, cross(cross(V, T), T), anisotropic)) with
    T rotated by aniso_rotation * 2 pi (shader.wgsl:2108-2116)."""
    n = np.array([0.0, 0.0, 1.0])
    V = np.array([0.3, 0.2, 1.0])
    V /= np.linalg.norm(V)
    aniso, rot = 0.8, 0.3
    up = np.array([0.0, 0.0, 1.0]) if abs(n[1]) > 0.99999 else np.array([0.0, 1.0, 0.0])
    T = np.cross(up, n)
    T /= np.linalg.norm(T)
    B = np.cross(n, T)
    ang = rot * 2 * math.pi
    T = T * math.cos(ang) + B * math.sin(ang)
    ns = n * (1 - aniso) + np.cross(np.cross(V, T), T) * aniso
    ns /= np.linalg.norm(ns)
    expect = -V + 2 * np.dot(V, ns) * ns           # reflect(-V, N_spec)
    mirror = -V + 2 * np.dot(V, n) * n
    mat = _material_bytes(anisotropic=aniso, anisotropicRotation=rot)
    for state in (12345, 777, 99991, 2024):
        cont, d, tp = oracle.sample_surface(mat, n, 0.0, 1.0, (1.0, 1.0, 1.0), V, state)
        assert cont
        assert np.dot(d, expect) > 1 - 1e-6
    assert np.dot(expect, mirror) < 0.99           # the tilt is large enough to matter


# ----------------------------------------------------------------------------- stale tangents
def stale_tangent_scene(with_plane: bool):
    """A normal-mapped triangle pair at z = 0 facing the camera, and (optionally) a plane at
    z = -5 behind it.  trace_scene tests planes before the TLAS (shader.wgsl:757-761), so the
    plane is accepted first and writes tangent (0, 1, 0) and bitangent (-1, 0, 0)
    (trace_plane: normalize(cross(n, x)), normalize(cross(n, t))); the triangle then wins
    without writing a frame."""
    texel = np.array([128, 200, 255, 255], np.uint8)
    tex = sc.Texture(np.tile(texel, (4, 4, 1)), "n")
    mat = sc.Material("mapped", [0.6, 0.6, 0.6], 0.5, normalTex=tex, normalMultiplier=1.0)
    quad = _model("quad", [[(-3.0, -3.0, 0.0), (3.0, -3.0, 0.0), (3.0, 3.0, 0.0)],
                           [(-3.0, -3.0, 0.0), (3.0, 3.0, 0.0), (-3.0, 3.0, 0.0)]])
    s = sc.Scene(8, 8)
    s.add(sc.Model("quad", mat, quad))
    if with_plane:
        s.add(sc.Plane("back", sc.Material("p", [0.3, 0.3, 0.3], 1.0), 0.0, 0.0, 1.0, -5.0))
    s.background = sc.HDRTexture([1.0, 1.0, 1.0])
    cam = s.camera
    cam.position = sc.gm.vec3(0.0, 0.0, 6.0)
    cam.target = sc.gm.vec3(0.0, 0.0, 0.0)
    cam.fov = 20.0
    cam.aspect = 1.0
    return s, texel


def stale_tangent_expected(texel, with_plane: bool):
    """get_surface_context's normal map (shader.wgsl:1399-1404) in float64, then gbuf_main's
    flip towards the viewer (2556)."""
    nm = texel[:3] / 255.0 * 2.0 - 1.0
    nm = nm / np.linalg.norm(nm)                    # multiplier 1: (m, m, 1) scaling is a no-op
    N = np.array([0.0, 0.0, 1.0])
    T = np.array([0.0, 1.0, 0.0]) if with_plane else np.zeros(3)
    B = np.array([-1.0, 0.0, 0.0]) if with_plane else np.zeros(3)
    v = T * nm[0] + B * nm[1] + N * nm[2]
    v /= np.linalg.norm(v)
    return v if v[2] > 0 else -v


def test_stale_tangent_frame_oracle():
    for with_plane in (True, False):
        s, texel = stale_tangent_scene(with_plane)
        packed = sc.pack_scene_data(s)
        s.camera.update_rays2()
        params = sc.pack_params(s, packed, 8, 8, 0, 1)
        g = np.zeros((8, 8, 12), np.float32)
        out = np.zeros((8, 8, 4), np.uint8)
        assert oracle.gbuffer(oracle.OracleScene(packed), params, (0, 0, 8, 8), g, out) == 0
        np.testing.assert_allclose(g[4, 4, :3], stale_tangent_expected(texel, with_plane), atol=1e-5)


@pytest.mark.gpu
def test_stale_tangent_frame_device():
    from webgpuraytracer_b200 import renderer as rd
    for with_plane in (True, False):
        s, texel = stale_tangent_scene(with_plane)
        r = rd.Renderer(8, 8)
        r.set_scene(s, isgbuf=True)
        r.render_gbuffer()
        g = r.read_gbuffer()
        r.close()
        np.testing.assert_allclose(g[4, 4, :3], stale_tangent_expected(texel, with_plane), atol=1e-5)
