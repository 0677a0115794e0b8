"""Seeded synthetic scenes with the shapes of the benchmark configurations.

No public scene or dataset is involved: every scene is generated here from a seed with the
reference's own PRNG (mulberry32, scene.js:665-672) and built with the scene classes of
scene.py, so the packed buffers are what tracer.js would produce for the same objects.

    small_scene      256x256, 16 spp, 4 bounces: 5 spheres, 2 cubes, 1 ground plane, constant
                     white environment (the reference's CPU-sized case)
    flagship_scene   1920x1080, 64 spp, 8 bounces: a noise-displaced icosphere (subdivision 6,
                     81,920 triangles) instanced 64x with similarity transforms, 32 spheres,
                     cylinders and tori with randomised Disney materials, and a 2048x1024 RLE
                     RGBE sky with a 0.5-degree sun of radiance 5e4 (importance sampled)
"""
from __future__ import annotations

import math
import struct
from dataclasses import dataclass

import numpy as np

from . import scene as sc


def mulberry32(a: int):
    """scene.js:665-672"""
    state = [a & 0xFFFFFFFF]

    def imul(x, y):
        return (x * y) & 0xFFFFFFFF

    def rnd() -> float:
        state[0] = (state[0] + 0x6D2B79F5) & 0xFFFFFFFF
        t = state[0]
        t = imul(t ^ (t >> 15), t | 1)
        t ^= (t + imul(t ^ (t >> 7), t | 61)) & 0xFFFFFFFF
        return ((t ^ (t >> 14)) & 0xFFFFFFFF) / 4294967296

    return rnd


@dataclass
class Config:
    name: str
    width: int
    height: int
    spp: int
    bounces: int


SMALL = Config("small-256x256-16spp-4b", 256, 256, 16, 4)
FLAGSHIP = Config("flagship-1920x1080-64spp-8b", 1920, 1080, 64, 8)


def _uniform(rnd, lo, hi):
    return lo + (hi - lo) * rnd()


def small_scene(seed: int = 1, width: int = 256, height: int = 256, bounces: int = 4) -> sc.Scene:
    """5 spheres (r ~ U[0.3,1]), 2 cubes (edge ~ U[0.5,1.5]), centres ~ U[-4,4]^3, a ground
    plane; each object gets a Lambertian, GGX-metal or dielectric material."""
    rnd = mulberry32(seed)
    s = sc.Scene(width, height)
    s.bounces = bounces

    def material(i):
        kind = int(rnd() * 3)
        if kind == 0:
            return sc.Material(f"lambert{i}", [_uniform(rnd, 0.1, 0.9) for _ in range(3)], 1.0, metallic=0.0)
        if kind == 1:
            return sc.Material(f"metal{i}", [_uniform(rnd, 0.1, 0.9) for _ in range(3)], _uniform(rnd, 0.05, 0.6),
                               metallic=1.0)
        return sc.Material(f"glass{i}", [_uniform(rnd, 0.7, 1.0) for _ in range(3)], 0.0, ior=1.5, transmission=1.0)

    for i in range(5):
        c = [_uniform(rnd, -4, 4) for _ in range(3)]
        s.add(sc.Sphere(f"sphere{i}", material(i), c[0], c[1], c[2], _uniform(rnd, 0.3, 1.0)))
    for i in range(2):
        c = [_uniform(rnd, -4, 4) for _ in range(3)]
        e = _uniform(rnd, 0.5, 1.5) / 2
        s.add(sc.Cube(f"cube{i}", material(5 + i), c[0] - e, c[1] - e, c[2] - e, c[0] + e, c[1] + e, c[2] + e))
    d = _uniform(rnd, -5.0, -4.0)
    s.add(sc.Plane("ground", material(7), 0, 1, 0, d))
    s.background = sc.HDRTexture([1.0, 1.0, 1.0])
    cam = s.camera
    cam.position = sc.gm.vec3(0.0, 3.0, 14.0)
    cam.target = sc.gm.vec3(0.0, 0.0, 0.0)
    cam.fov = 45.0
    cam.aperture = 0.0
    cam.exposure = 1.0
    cam.aspect = width / height
    return s


# ----------------------------------------------------------------------------- meshes
def icosphere(subdivisions: int):
    """Unit icosphere: (positions float64 [V,3], faces int64 [F,3]); F = 20 * 4^subdivisions."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
         (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
         (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    verts = np.array(v, dtype=np.float64)
    verts /= np.linalg.norm(verts, axis=1, keepdims=True)
    faces = np.array(f, dtype=np.int64)
    for _ in range(subdivisions):
        e = np.concatenate([faces[:, [0, 1]], faces[:, [1, 2]], faces[:, [2, 0]]])
        e.sort(axis=1)
        uniq, inv = np.unique(e, axis=0, return_inverse=True)
        inv = inv.reshape(-1)
        mid = verts[uniq[:, 0]] + verts[uniq[:, 1]]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        base = len(verts)
        verts = np.concatenate([verts, mid])
        nf = len(faces)
        a = base + inv[:nf]
        b = base + inv[nf:2 * nf]
        c = base + inv[2 * nf:]
        f0, f1, f2 = faces[:, 0], faces[:, 1], faces[:, 2]
        faces = np.concatenate([np.stack([f0, a, c], 1), np.stack([f1, b, a], 1), np.stack([f2, c, b], 1),
                                np.stack([a, b, c], 1)])
    return verts, faces


def value_noise3(p: np.ndarray, seed: int) -> np.ndarray:
    """Smooth 3-D lattice value noise in [-1, 1] (integer hash at lattice points, smoothstep)."""
    def h(ix, iy, iz):
        n = (ix * 73856093) ^ (iy * 19349663) ^ (iz * 83492791) ^ (seed * 2654435761)
        n = n & 0xFFFFFFFF
        n = (n ^ (n >> 13)) * 1274126177 & 0xFFFFFFFF
        n = n ^ (n >> 16)
        return (n & 0xFFFFFF) / float(0xFFFFFF) * 2.0 - 1.0

    fl = np.floor(p)
    i = fl.astype(np.int64)
    fr = p - fl
    w = fr * fr * (3 - 2 * fr)
    out = np.zeros(len(p))
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                val = h(i[:, 0] + dx, i[:, 1] + dy, i[:, 2] + dz)
                wx = w[:, 0] if dx else 1 - w[:, 0]
                wy = w[:, 1] if dy else 1 - w[:, 1]
                wz = w[:, 2] if dz else 1 - w[:, 2]
                out += val * wx * wy * wz
    return out


def displaced_icosphere(subdivisions: int = 6, amplitude: float = 0.1, seed: int = 1) -> sc.ModelData:
    """Icosphere with every vertex moved along its normal by amplitude x 3-octave value noise;
    area-weighted smooth normals (calculateSmoothNormals) and spherical UVs."""
    verts, faces = icosphere(subdivisions)
    noise = np.zeros(len(verts))
    amp, freq = 1.0, 2.0
    for octave in range(3):
        noise += amp * value_noise3(verts * freq, seed + octave)
        amp *= 0.5
        freq *= 2.0
    pos = verts * (1.0 + amplitude * noise)[:, None]
    pos32 = pos.astype(np.float32)
    p = pos32.astype(np.float64)
    fn = np.cross(p[faces[:, 1]] - p[faces[:, 0]], p[faces[:, 2]] - p[faces[:, 0]])
    nrm = np.zeros_like(p)
    for k in range(3):
        np.add.at(nrm, faces[:, k], fn)
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    r = np.linalg.norm(p, axis=1)
    uv = np.stack([np.arctan2(p[:, 2], p[:, 0]) / (2 * math.pi) + 0.5, np.arcsin(p[:, 1] / r) / math.pi + 0.5], 1)
    md = sc.ModelData(f"icosphere{subdivisions}", pos32, nrm.astype(np.float32), uv.astype(np.float32), faces)
    return md.generate_bvh()


# ----------------------------------------------------------------------------- environment
def procedural_sky(width: int = 2048, height: int = 1024, sun_radiance: float = 5e4,
                   sun_elevation_deg: float = 35.0, sun_azimuth_deg: float = 60.0,
                   sun_diameter_deg: float = 0.5) -> np.ndarray:
    """Equirectangular sky (rows top to bottom in the layout sample_sky reads): a horizon to
    zenith gradient, a darker ground below the horizon, and a sun disc."""
    u = (np.arange(width) + 0.5) / width
    v = (np.arange(height) + 0.5) / height
    phi = (u - 0.5) * 2 * math.pi                       # sample_sky: u = 0.5 + atan2(z, x) / 2pi
    theta = (0.5 - v) * math.pi                         # v = 0.5 - asin(y) / pi
    ph, th = np.meshgrid(phi, theta)
    dx, dy, dz = np.cos(th) * np.cos(ph), np.sin(th), np.cos(th) * np.sin(ph)
    elev = np.clip(dy, 0.0, 1.0)
    horizon = np.array([1.0, 0.9, 0.8])
    zenith = np.array([0.25, 0.45, 1.0])
    g = np.sqrt(elev)[..., None]
    sky = horizon * (1 - g) + zenith * g
    ground = np.array([0.3, 0.26, 0.22]) * 0.5
    sky = np.where((dy < 0)[..., None], ground, sky)
    se, sa = math.radians(sun_elevation_deg), math.radians(sun_azimuth_deg)
    sun = np.array([math.cos(se) * math.cos(sa), math.sin(se), math.cos(se) * math.sin(sa)])
    cosang = dx * sun[0] + dy * sun[1] + dz * sun[2]
    disc = cosang >= math.cos(math.radians(sun_diameter_deg / 2))
    sky[disc] = np.array([1.0, 0.96, 0.9]) * sun_radiance
    return sky.astype(np.float32)


def encode_rgbe(img: np.ndarray) -> bytes:
    """Radiance .hdr writer (new-style run-length encoded scanlines)."""
    h, w, _ = img.shape
    v = img.max(axis=2).astype(np.float64)
    m, e = np.frexp(v)
    scale = np.where(v > 1e-32, m * 256.0 / np.where(v > 0, v, 1), 0.0)
    rgbe = np.zeros((h, w, 4), dtype=np.uint8)
    rgbe[..., :3] = np.clip(np.floor(img * scale[..., None]), 0, 255).astype(np.uint8)
    rgbe[..., 3] = np.where(v > 1e-32, e + 128, 0).astype(np.uint8)
    out = bytearray(b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n-Y %d +X %d\n" % (h, w))
    for y in range(h):
        out += bytes([2, 2, w >> 8, w & 255])
        for ch in range(4):
            row = rgbe[y, :, ch]
            i = 0
            while i < w:
                # run of equal bytes
                j = i
                while j < w and j - i < 127 and row[j] == row[i]:
                    j += 1
                if j - i >= 3:
                    out += bytes([128 + (j - i), int(row[i])])
                    i = j
                    continue
                # literal chunk until the next run of 3 or 128 bytes
                k = i
                while k < w and k - i < 128:
                    if k + 2 < w and row[k] == row[k + 1] == row[k + 2]:
                        break
                    k += 1
                if k == i:
                    k = i + 1
                out += bytes([k - i]) + row[i:k].tobytes()
                i = k
    return bytes(out)


_SKY_CACHE: dict = {}


def flagship_sky() -> sc.HDRTexture:
    key = "flagship"
    if key not in _SKY_CACHE:
        _SKY_CACHE[key] = encode_rgbe(procedural_sky())
    return sc.HDRTexture.from_rgbe(_SKY_CACHE[key], exposure=1.0)


def _disney_material(rnd, name):
    return sc.Material(
        name, [_uniform(rnd, 0.1, 0.9) for _ in range(3)], _uniform(rnd, 0.0, 1.0),
        metallic=_uniform(rnd, 0, 1), ior=_uniform(rnd, 1.0, 2.5), specularTint=_uniform(rnd, 0, 1),
        anisotropic=_uniform(rnd, 0, 1), anisotropicRotation=_uniform(rnd, 0, 1), sheen=_uniform(rnd, 0, 1),
        sheenTint=_uniform(rnd, 0, 1), clearcoat=_uniform(rnd, 0, 1), clearcoatGloss=_uniform(rnd, 0, 1),
        clearcoatIor=_uniform(rnd, 1.0, 2.0), transmission=_uniform(rnd, 0, 1), subsurface=_uniform(rnd, 0, 1),
        concentration=_uniform(rnd, 0.0, 2.0))


def _random_rotation(rnd):
    """Uniform random rotation (Shoemake) as axis and angle for Primitive.rotate."""
    u1, u2, u3 = rnd(), rnd(), rnd()
    q = (math.sqrt(1 - u1) * math.sin(2 * math.pi * u2), math.sqrt(1 - u1) * math.cos(2 * math.pi * u2),
         math.sqrt(u1) * math.sin(2 * math.pi * u3), math.sqrt(u1) * math.cos(2 * math.pi * u3))
    if q[3] < 0:
        q = tuple(-c for c in q)
    s = math.sqrt(q[0] ** 2 + q[1] ** 2 + q[2] ** 2)
    if s < 1e-9:
        return 0.0, (0.0, 1.0, 0.0)
    return 2 * math.acos(min(1.0, q[3])), (q[0] / s, q[1] / s, q[2] / s)


_MESH_CACHE: dict = {}


def flagship_mesh(subdivisions: int = 6) -> sc.ModelData:
    if subdivisions not in _MESH_CACHE:
        _MESH_CACHE[subdivisions] = displaced_icosphere(subdivisions, 0.1, seed=7)
    return _MESH_CACHE[subdivisions]


def flagship_scene(seed: int = 1, width: int = 1920, height: int = 1080, bounces: int = 8,
                   instances: int = 64, prims: int = 32, subdivisions: int = 6, sky: bool = True) -> sc.Scene:
    """The two-level-BVH, full-Disney-BSDF, importance-sampled-environment workload."""
    rnd = mulberry32(seed)
    s = sc.Scene(width, height)
    s.bounces = bounces
    mesh = flagship_mesh(subdivisions)
    for i in range(instances):
        m = sc.Model(f"blob{i}", _disney_material(rnd, f"blob_mat{i}"), mesh)
        scale = _uniform(rnd, 0.3, 1.2)
        theta, axis = _random_rotation(rnd)
        m.position = sc.gm.vec3(_uniform(rnd, -10, 10), _uniform(rnd, 0.0, 5.0), _uniform(rnd, -10, 10))
        m.scale = sc.gm.vec3(scale, scale, scale)
        m.rotate(theta, *axis)
        s.add(m)
    for i in range(prims):
        mat = _disney_material(rnd, f"prim_mat{i}")
        kind = i % 3
        pos = (_uniform(rnd, -10, 10), _uniform(rnd, 0.0, 5.0), _uniform(rnd, -10, 10))
        if kind == 0:
            s.add(sc.Sphere(f"sphere{i}", mat, pos[0], pos[1], pos[2], _uniform(rnd, 0.3, 1.2)))
        elif kind == 1:
            c = sc.Cylinder(f"cylinder{i}", mat, _uniform(rnd, 0.0, 1.0))
            r, hgt = _uniform(rnd, 0.3, 1.0), _uniform(rnd, 0.5, 2.0)
            theta, axis = _random_rotation(rnd)
            c.position = sc.gm.vec3(*pos)
            c.scale = sc.gm.vec3(r, hgt, r)
            c.rotate(theta, *axis)
            s.add(c)
        else:
            outer = _uniform(rnd, 0.5, 1.2)
            t = sc.Torus(f"torus{i}", mat, outer, outer * _uniform(rnd, 0.1, 0.5))
            theta, axis = _random_rotation(rnd)
            t.position = sc.gm.vec3(*pos)
            t.rotate(theta, *axis)
            s.add(t)
    s.background = flagship_sky() if sky else sc.HDRTexture([1.0, 1.0, 1.0])
    cam = s.camera
    cam.position = sc.gm.vec3(0.0, 7.0, 24.0)
    cam.target = sc.gm.vec3(0.0, 2.0, 0.0)
    cam.fov = 45.0
    cam.aperture = 0.0
    cam.exposure = 1.0
    cam.aspect = width / height
    return s


# ----------------------------------------------------------------------------- textured scenes
def texture_set(size: int = 64, seed: int = 1) -> dict[str, sc.Texture]:
    """Seeded rgba8 images at one common size: an albedo whose alpha mixes fully transparent,
    partly covered and opaque cells; a tangent-space normal map of sinusoidal bumps; a height
    field (red) of rounded tiles; roughness (green), metallic (blue) and emissive images of
    value noise."""
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:size, 0:size].astype(np.float64) / size
    albedo = np.empty((size, size, 4), np.uint8)
    albedo[..., :3] = rng.integers(40, 256, (size, size, 3))
    cells = ((x * 8).astype(int) + (y * 8).astype(int) * 3) % 4
    albedo[..., 3] = np.array([0, 77, 200, 255], np.uint8)[cells]
    hx = 0.35 * np.cos(2 * math.pi * 3 * x) * np.sin(2 * math.pi * 2 * y)
    hy = 0.35 * np.sin(2 * math.pi * 3 * x) * np.cos(2 * math.pi * 2 * y)
    n = np.stack([-hx, -hy, np.ones_like(hx)], -1)
    n /= np.linalg.norm(n, axis=-1, keepdims=True)
    normal = np.empty((size, size, 4), np.uint8)
    normal[..., :3] = np.clip(np.round((n * 0.5 + 0.5) * 255), 0, 255).astype(np.uint8)
    normal[..., 3] = 255

    tile = np.sin(math.pi * ((x * 4) % 1.0)) * np.sin(math.pi * ((y * 4) % 1.0))
    height = np.full((size, size, 4), 255, np.uint8)
    height[..., :3] = 0
    height[..., 0] = np.clip(np.round(np.sqrt(np.maximum(tile, 0.0)) * 255), 0, 255).astype(np.uint8)

    def noise_image(channel):
        img = np.full((size, size, 4), 255, np.uint8)
        img[..., :3] = 0
        img[..., channel] = rng.integers(0, 256, (size, size))
        return img

    emissive = np.full((size, size, 4), 255, np.uint8)
    emissive[..., :3] = (rng.random((size, size, 1)) * np.array([255, 200, 120])).astype(np.uint8)
    return {"albedo": sc.Texture(albedo, "albedo"), "normal": sc.Texture(normal, "normal"),
            "height": sc.Texture(height, "height"),
            "roughness": sc.Texture(noise_image(1), "roughness"), "metallic": sc.Texture(noise_image(2), "metallic"),
            "emissive": sc.Texture(emissive, "emissive")}


def textured_scene(seed: int = 1, width: int = 128, height: int = 128, bounces: int = 6, tex_size: int = 64,
                   sky: bool = True, pom: bool = False) -> sc.Scene:
    """Every primitive kind with textured materials: alpha cut-outs (albedo alpha) on a sphere,
    a cube, a mesh instance, a listed mesh and a plane, so shadow rays cross partly covered
    surfaces; normal maps on a cube, a torus and meshes (triangles and tori keep the tangent frame
    of an earlier closest candidate); roughness and metallic maps on a cylinder; an emissive map;
    a sphere and a box light sampled explicitly, and an importance-sampled sky.  With `pom`, the
    ground, the bumpy material and a cube also carry height fields (parallax occlusion mapping:
    a depth map and an inverted height map with different layer counts and offsets)."""
    rnd = mulberry32(seed)
    t = texture_set(tex_size, seed)
    s = sc.Scene(width, height)
    s.bounces = bounces
    cut = sc.Material("cutout", [0.9, 0.8, 0.7], 0.8, albedoTex=t["albedo"], uvScale=[2.0, 1.0])
    bumpy = sc.Material("bumpy", [0.6, 0.7, 0.9], 0.3, metallic=0.3, normalTex=t["normal"], normalMultiplier=1.5)
    rough = sc.Material("rough", [0.8, 0.5, 0.3], 0.9, metallic=1.0, roughnessTex=t["roughness"],
                        metallicTex=t["metallic"], clearcoat=0.5)
    glow = sc.Material("glow", [1, 1, 1], 1.0, emittance=[1.0, 0.8, 0.6], emissionIntensity=2.0, emissiveTex=t["emissive"])
    all_in = sc.Material("all", [0.7, 0.7, 0.7], 0.5, albedoTex=t["albedo"], normalTex=t["normal"],
                         roughnessTex=t["roughness"], uvScale=[3.0, 3.0])
    ground = sc.Material("ground", [0.8, 0.8, 0.8], 0.7, albedoTex=t["albedo"], normalTex=t["normal"],
                         uvScale=[0.25, 0.25])
    if pom:
        ground.heightTex = t["height"]
        ground.heightMultiplier, ground.heightSamp, ground.heightOffset = 0.08, 24, 0.5
        bumpy.heightTex = t["height"]
        bumpy.heightMultiplier, bumpy.heightSamp = -0.05, 12
    s.add(sc.Sphere("cut_sphere", cut, _uniform(rnd, -2.5, -1.5), 0.5, 0.0, 1.0))
    s.add(sc.Cube("cut_cube", all_in, 0.5, -1.0, -1.5, 1.7, 0.2, -0.3))
    if pom:
        s.add(sc.Cube("relief_cube", sc.Material("relief", [0.5, 0.8, 0.5], 0.4, heightTex=t["height"],
                                                 heightMultiplier=0.1, heightSamp=40, uvScale=[2.0, 2.0]),
                      2.4, -2.0, -1.8, 3.4, -1.0, -0.8))
    s.add(sc.Cube("bump_cube", bumpy, -0.6, -1.9, 1.0, 0.4, -0.9, 2.0))
    tor = s.add(sc.Torus("bump_torus", bumpy, 1.0, 0.35))
    tor.set_position(2.2, 0.6, 1.0)
    tor.rotate(0.7, 1, 0, 0)
    cyl = sc.Cylinder("rough_cyl", rough, 0.6)
    cyl.position = sc.gm.vec3(-0.5, -2.0, -2.5)
    cyl.scale = sc.gm.vec3(0.8, 2.0, 0.8)
    s.add(cyl)
    s.add(sc.Sphere("glow_sphere", glow, 0.0, 2.3, -1.0, 0.4))
    mesh = displaced_icosphere(2, 0.15, seed=seed)
    m1 = s.add(sc.Model("cut_mesh", all_in, mesh))
    m1.position = sc.gm.vec3(-1.2, -1.2, 2.2)
    m1.scale = sc.gm.vec3(0.8, 0.8, 0.8)
    m2 = s.add(sc.Model("bump_list_mesh", bumpy, mesh, in_scene_bvh=False))
    m2.position = sc.gm.vec3(1.6, -1.4, 2.6)
    m2.scale = sc.gm.vec3(0.6, 0.6, 0.6)
    s.add(sc.Plane("ground", ground, 0, 1, 0, -2.0))
    lamp = sc.Material("lamp", [1, 0.9, 0.8], 1.0, emittance=[1, 0.9, 0.7], emissionIntensity=8.0)
    a = s.add(sc.Sphere("lamp0", lamp, 0.8, 4.0, 1.5, 0.5))
    a.enableNEE = True
    b = s.add(sc.Cube("lamp1", lamp, -3.0, 3.0, -2.0, -2.2, 3.5, -1.4))
    b.enableNEE = True
    if sky:
        s.background = sc.HDRTexture.from_rgbe(encode_rgbe(procedural_sky(256, 128, sun_radiance=2e3,
                                                                          sun_diameter_deg=3.0)), exposure=1.0)
    else:
        s.background = sc.HDRTexture([1.0, 1.0, 1.0])
    cam = s.camera
    cam.position = sc.gm.vec3(0.0, 2.0, 9.0)
    cam.target = sc.gm.vec3(0.0, -0.5, 0.0)
    cam.fov = 50.0
    cam.aperture = 0.0
    cam.exposure = 1.0
    cam.aspect = width / height
    return s


BATCH_SIZES = ((256, 256), (512, 512), (1280, 720), (1920, 1080))
BATCH_SPP = (4, 16, 64)


def batch_scene(seed: int = 1, bounces: int = 8) -> sc.Scene:
    """The batched-views workload's scene: the displaced icosphere at 7 subdivisions (327,680
    triangles, the icosphere level nearest above a 262,144-triangle mesh) instanced 16 times
    (5.24 M triangles) plus 64 analytic primitives, under the importance-sampled procedural sky."""
    return flagship_scene(seed, 1920, 1080, bounces, instances=16, prims=64, subdivisions=7)


def batch_views(seed: int = 1, n: int = 32) -> list[dict]:
    """n camera views with seeded sizes (uniform over BATCH_SIZES), samples (uniform over
    BATCH_SPP) and positions on a ring around the scene, looking at its centre region."""
    rnd = mulberry32(seed * 7919 + 17)
    views = []
    for i in range(n):
        w, h = BATCH_SIZES[min(int(rnd() * len(BATCH_SIZES)), len(BATCH_SIZES) - 1)]
        spp = BATCH_SPP[min(int(rnd() * len(BATCH_SPP)), len(BATCH_SPP) - 1)]
        ang = rnd() * 2.0 * math.pi
        radius = _uniform(rnd, 16.0, 26.0)
        eye = (radius * math.cos(ang), _uniform(rnd, 2.0, 10.0), radius * math.sin(ang))
        target = (_uniform(rnd, -3, 3), _uniform(rnd, 0.5, 3.0), _uniform(rnd, -3, 3))
        views.append({"width": w, "height": h, "spp": spp, "eye": eye, "target": target})
    return views


def view_params(scene: sc.Scene, packed, view: dict, frame: int = 0, seed: int = 1) -> np.ndarray:
    """The 112-byte SceneParams of one view: the scene's camera moved to the view's eye and
    target, with the view's aspect ratio."""
    cam = scene.camera
    cam.position = sc.gm.vec3(*view["eye"])
    cam.target = sc.gm.vec3(*view["target"])
    cam.aspect = view["width"] / view["height"]
    cam.update_rays2()
    return sc.pack_params(scene, packed, view["width"], view["height"], frame, seed)
