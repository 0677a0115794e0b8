"""Scene model and buffer packing of tracer.js, restated for the native renderer.

Classes mirror tracer.js's (Material 208-297, Primitive/Sphere/Cube/Cylinder/Torus/Plane
320-910, ModelData/Model 912-1417, Camera 1419-1507, SceneBVHBuilder 1509-1619, Scene 1621-1690,
Light 1692-1711, HDRTexture 22-205) and pack_scene_data mirrors Renderer.packSceneData
(1819-1917): the result is the set of byte buffers the WGSL bind group receives, which
wgpt_upload_scene takes unchanged.  Matrix and vector arithmetic uses gl-matrix semantics
(glmat.py); the BVH and CDF builders are the native ones in libwgpt.so.
"""
from __future__ import annotations

import ctypes as C
import math
import struct
from dataclasses import dataclass, field

import numpy as np

from . import glmat as gm
from ._lib import (HAS_CUBES, HAS_CYLINDERS, HAS_HEIGHTMAPS, HAS_LIGHTS, HAS_LIST_MESHES, HAS_MESHES,
                   HAS_PLANES, HAS_SKYBOX, HAS_SPHERES, HAS_TORI, MIS_SKYBOX, check, lib, ptr)

SIZES = {"vec2f": 8, "vec3f": 12, "vec4f": 16, "f32": 4, "i32": 4, "u32": 4, "mat2x2f": 16, "mat3x3f": 36,
         "mat4x4f": 64}


def _js_or(v, default):
    """JavaScript `v || default`: falsy values (undefined, 0, NaN) take the default."""
    if v is None or v == 0 or (isinstance(v, float) and math.isnan(v)):
        return default
    return v


# ----------------------------------------------------------------------------- environment
def double_to_half_bits(x: float) -> int:
    """Float16Array store of a double (round to nearest even)."""
    return int(np.array([x], dtype=np.float64).astype(np.float16).view(np.uint16)[0])


class HDRTexture:
    """tracer.js:22-205.  `data` holds width*height*4 IEEE halves (as uint16)."""

    def __init__(self, color=None, exposure: float = 1.0, rgba16f: np.ndarray | None = None,
                 width: int = 1, height: int = 1):
        self.exposure = exposure
        self.threshold = 65536 - 16 - 1
        self.enableNEE = True
        if rgba16f is None:
            c = color if color is not None else [0.02, 0.03, 0.05, 1.0]
            self.width = self.height = 1
            # new Float16Array([r, g, b, 1]) -- doubles rounded straight to half (exact for
            # float16-representable inputs; numpy converts through float64 -> float16 here)
            self.data = np.array([c[0], c[1], c[2], 1.0], dtype=np.float64).astype(np.float16).view(np.uint16)
            self.plainColor = True
        else:
            self.width, self.height = int(width), int(height)
            self.data = np.ascontiguousarray(rgba16f, dtype=np.uint16).reshape(-1)
            assert self.data.size == self.width * self.height * 4
            self.plainColor = False

    @classmethod
    def from_rgbe(cls, file_bytes: bytes, exposure: float = 1.0) -> "HDRTexture":
        """HDRTexture._load + parseHdr + updateData through the native decoder."""
        L = lib()
        buf = np.frombuffer(file_bytes, dtype=np.uint8)
        w, h = C.c_uint32(0), C.c_uint32(0)
        check(L.wgpt_decode_rgbe(ptr(buf), buf.size, exposure, None, C.byref(w), C.byref(h)), "decode_rgbe")
        out = np.zeros(w.value * h.value * 4, dtype=np.uint16)
        check(L.wgpt_decode_rgbe(ptr(buf), buf.size, exposure, ptr(out), C.byref(w), C.byref(h)), "decode_rgbe")
        return cls(exposure=exposure, rgba16f=out, width=w.value, height=h.value)

    def build_hdr_cdf(self) -> tuple[np.ndarray, int, float]:
        """buildHDRCDF: (skyCDF float32, sky_cdf_index, totalWeight)."""
        n = (self.height + 1) + self.height * (self.width + 1)
        cdf = np.zeros(n, dtype=np.float32)
        total = C.c_double(0)
        check(lib().wgpt_build_env_cdf(ptr(self.data), self.width, self.height, self.exposure, ptr(cdf),
                                       C.byref(total)), "build_env_cdf")
        return cdf, self.height + 1, total.value

    def build_env_alias(self) -> np.ndarray:
        """Alias table over buildHDRCDF's texel weights (FP64): (width * height, 2) uint32 rows of
        (float32 probability bits, alias texel), the layout of wgpt_scene_desc.sky_alias."""
        n = self.width * self.height
        prob = np.zeros(n, dtype=np.float32)
        alias = np.zeros(n, dtype=np.uint32)
        check(lib().wgpt_build_env_alias(ptr(self.data), self.width, self.height, self.exposure, ptr(prob),
                                         ptr(alias)), "build_env_alias")
        return np.ascontiguousarray(np.stack([prob.view(np.uint32), alias], axis=1))


# ----------------------------------------------------------------------------- materials
class Texture:
    """tracer.js:5-20: one image of the texture array.  `image` is (H, W, 4) uint8 rgba, already at
    the array's common size (prepareTextureArray, tracer.js:1919-1953, resizes every texture to
    512 x 512 in the browser); texIndex is its layer once a scene is packed."""

    def __init__(self, image, name: str = "New Texture"):
        self.name = name
        self.image = np.ascontiguousarray(image, dtype=np.uint8)
        assert self.image.ndim == 3 and self.image.shape[2] == 4, "texture images are (H, W, 4) rgba8"
        self.texIndex = -1


TEXTURE_SLOTS = ("emissiveTex", "albedoTex", "normalTex", "heightTex", "roughnessTex", "metallicTex")


class Material:
    """tracer.js:208-256"""

    def __init__(self, name="New Material", color=(1, 1, 1), roughness=0.5, **o):
        self.name = name
        self.color = list(color)
        self.roughness = roughness
        self.metallic = o["metallic"] if o.get("metallic") is not None else 0.0
        self.ior = _js_or(o.get("ior"), 1.5)
        self.emittance = list(_js_or(o.get("emittance"), [1, 1, 1]))
        self.emissionIntensity = _js_or(o.get("emissionIntensity"), 0.0)
        self.subsurface = _js_or(o.get("subsurface"), 0.0)
        self.subsurfaceTint = list(_js_or(o.get("subsurfaceTint"), list(self.color)))
        self.specularTint = _js_or(o.get("specularTint"), 0.0)
        self.anisotropic = _js_or(o.get("anisotropic"), 0.0)
        self.anisotropicRotation = _js_or(o.get("anisotropicRotation"), 0.0)
        self.sheen = _js_or(o.get("sheen"), 0.0)
        self.sheenTint = _js_or(o.get("sheenTint"), 0.5)
        self.clearcoat = _js_or(o.get("clearcoat"), 0.0)
        self.clearcoatGloss = _js_or(o.get("clearcoatGloss"), 1.0)
        self.clearcoatIor = _js_or(o.get("clearcoatIor"), 1.5)
        self.transmission = _js_or(o.get("transmission"), 0.0)
        self.concentration = _js_or(o.get("concentration"), 1.0)
        self.uvScale = list(_js_or(o.get("uvScale"), [1, 1]))
        self.normalMultiplier = _js_or(o.get("normalMultiplier"), 1.0)
        self.heightMultiplier = o["heightMultiplier"] if o.get("heightMultiplier") is not None else 0.05
        self.heightSamp = _js_or(o.get("heightSamp"), 32)
        self.heightOffset = _js_or(o.get("heightOffset"), 0.0)
        for slot in TEXTURE_SLOTS:
            setattr(self, slot, o.get(slot) or None)
        self._index = -1

    def schema(self):
        """Material.getSchema (tracer.js:258-297)."""
        m = self
        idx = lambda t: t.texIndex if t is not None else -1
        return [
            ("vec3f", [v ** 2.2 for v in m.color]), ("f32", m.metallic),
            ("f32", m.roughness), ("f32", m.ior), ("f32", m.specularTint), ("f32", m.anisotropic),
            ("f32", m.anisotropicRotation), ("f32", m.sheen), ("f32", m.sheenTint), ("f32", m.clearcoat),
            ("f32", m.clearcoatGloss), ("f32", m.clearcoatIor), ("f32", m.transmission), ("f32", m.concentration),
            ("vec3f", [v ** 2.2 for v in m.subsurfaceTint]), ("f32", m.subsurface),
            ("vec3f", [v * m.emissionIntensity for v in m.emittance]), ("i32", idx(m.emissiveTex)),
            ("i32", idx(m.albedoTex)), ("i32", idx(m.normalTex)), ("i32", idx(m.heightTex)),
            ("i32", idx(m.roughnessTex)), ("i32", idx(m.metallicTex)), ("pad", None),
            ("vec2f", m.uvScale),
            ("vec4f", [m.normalMultiplier, m.heightMultiplier, m.heightSamp, m.heightOffset]),
        ]


# ----------------------------------------------------------------------------- primitives
class Primitive:
    """tracer.js:320-425"""
    type = "Primitive"

    def __init__(self, name, material):
        self.name = name
        self.material = material
        self.position = gm.vec3()
        self.scale = gm.vec3(1, 1, 1)
        self.rotation = gm.quat_identity()
        self.matrix = np.eye(4, dtype=np.float32).reshape(-1)
        self.invMatrix = np.eye(4, dtype=np.float32).reshape(-1)
        self.enableNEE = False
        self.lightIdx = -1

    def update_matrix(self):
        self.matrix = gm.mat4_from_rts(self.rotation, self.position, self.scale)
        self.invMatrix = gm.mat4_invert(self.matrix)

    def set_position(self, x, y, z):
        self.position = gm.vec3(x, y, z)
        self.update_matrix()
        return self

    def scale_set(self, x, y=None, z=None):
        if y is None:
            y = z = x
        self.scale = gm.vec3(x, y, z)
        self.update_matrix()
        return self

    def rotate(self, theta, ax, ay, az):
        """Primitive.rotate: setAxisAngle around the normalised axis (replaces the rotation)."""
        axis = gm.vec3_normalize(gm.vec3(ax, ay, az))
        self.rotation = gm.quat_set_axis_angle(axis, theta)
        self.update_matrix()
        return self

    def get_bounds(self):
        world = gm.mat4_invert(self.invMatrix)
        return transform_aabb([-1, -1, -1], [1, 1, 1], world)

    def get_area(self):
        return 0.0


def transform_aabb(lo, hi, m):
    """transformAABB (tracer.js:299-317)"""
    mn = gm.vec3(math.inf, math.inf, math.inf)
    mx = gm.vec3(-math.inf, -math.inf, -math.inf)
    for x in (lo[0], hi[0]):
        for y in (lo[1], hi[1]):
            for z in (lo[2], hi[2]):
                p = gm.vec3_transform_mat4(gm.vec3(x, y, z), m)
                mn = gm.vec3_min(mn, p)
                mx = gm.vec3_max(mx, p)
    return mn, mx


def _object_schema(o, type_id: int, param0: tuple[str, object]):
    return [("mat4x4f", o.invMatrix), ("i32", o.material._index), ("i32", o.lightIdx), ("i32", type_id),
            param0, ("vec3f", o.position), ("pad", None)]


class Sphere(Primitive):
    """tracer.js:427-489"""
    type = "Sphere"

    def __init__(self, name, material, x=0.0, y=0.0, z=0.0, radius=1.0):
        super().__init__(name, material)
        self.position = gm.vec3(x, y, z)
        self.scale = gm.vec3(radius, radius, radius)
        self.update_matrix()

    def get_area(self):
        r = (float(self.scale[0]) + float(self.scale[1]) + float(self.scale[2])) / 3
        return 4 * math.pi * r * r

    def get_bounds(self):
        m = [float(v) for v in self.matrix]
        ex = math.sqrt(m[0] * m[0] + m[4] * m[4] + m[8] * m[8])
        ey = math.sqrt(m[1] * m[1] + m[5] * m[5] + m[9] * m[9])
        ez = math.sqrt(m[2] * m[2] + m[6] * m[6] + m[10] * m[10])
        c = (m[12], m[13], m[14])
        return gm.f32([c[0] - ex, c[1] - ey, c[2] - ez]), gm.f32([c[0] + ex, c[1] + ey, c[2] + ez])

    def schema(self):
        return _object_schema(self, 1, ("pad", None))


class Cube(Primitive):
    """tracer.js:491-536"""
    type = "Cube"

    def __init__(self, name, material, minX=-1.0, minY=-1.0, minZ=-1.0, maxX=1.0, maxY=1.0, maxZ=1.0):
        super().__init__(name, material)
        self.position = gm.vec3((minX + maxX) / 2, (minY + maxY) / 2, (minZ + maxZ) / 2)
        self.scale = gm.vec3((maxX - minX) / 2, (maxY - minY) / 2, (maxZ - minZ) / 2)
        self.update_matrix()

    def get_area(self):
        s = [float(v) for v in self.scale]
        return 8 * (s[0] * s[1] + s[1] * s[2] + s[0] * s[2])

    def schema(self):
        return _object_schema(self, 2, ("pad", None))


class Cylinder(Primitive):
    """tracer.js:538-683; top_radius is the ratio of the top radius to the base radius."""
    type = "Cylinder"

    def __init__(self, name, material, top_radius=0.5):
        super().__init__(name, material)
        self.top_radius = top_radius

    def get_bounds(self):
        m = [float(v) for v in self.matrix]

        def circle(y_local, radius):
            ex = math.sqrt((radius * m[0]) ** 2 + (radius * m[8]) ** 2)
            ey = math.sqrt((radius * m[1]) ** 2 + (radius * m[9]) ** 2)
            ez = math.sqrt((radius * m[2]) ** 2 + (radius * m[10]) ** 2)
            wc = [float(v) for v in gm.vec3_transform_mat4(gm.vec3(0, y_local, 0), self.matrix)]
            return (gm.f32([wc[0] - ex, wc[1] - ey, wc[2] - ez]), gm.f32([wc[0] + ex, wc[1] + ey, wc[2] + ez]))

        b = circle(0, 1)
        t = circle(1, self.top_radius)
        return gm.vec3_min(b[0], t[0]), gm.vec3_max(b[1], t[1])

    def schema(self):
        return _object_schema(self, 3, ("f32", self.top_radius))


class Torus(Primitive):
    """tracer.js:685-785; the major radius is 1 in local space, inner_radius is the ratio."""
    type = "Torus"

    def __init__(self, name, material, outer=1.0, inner=0.3):
        super().__init__(name, material)
        self.scale_set(outer, outer, outer)
        self.inner_radius = inner / outer

    def get_bounds(self):
        m = [float(v) for v in self.matrix]
        R, r = 1.0, self.inner_radius
        ex = math.sqrt((R * m[0]) ** 2 + (R * m[8]) ** 2)
        ey = math.sqrt((R * m[1]) ** 2 + (R * m[9]) ** 2)
        ez = math.sqrt((R * m[2]) ** 2 + (R * m[10]) ** 2)
        wc = [float(v) for v in gm.vec3_transform_mat4(gm.vec3(0, 0, 0), self.matrix)]
        sx = math.sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2])
        sy = math.sqrt(m[4] * m[4] + m[5] * m[5] + m[6] * m[6])
        sz = math.sqrt(m[8] * m[8] + m[9] * m[9] + m[10] * m[10])
        th = r * max(sx, sy, sz)
        return (gm.f32([wc[0] - ex - th, wc[1] - ey - th, wc[2] - ez - th]),
                gm.f32([wc[0] + ex + th, wc[1] + ey + th, wc[2] + ez + th]))

    def schema(self):
        return _object_schema(self, 4, ("f32", self.inner_radius))


class Plane(Primitive):
    """tracer.js:787-910"""
    type = "Plane"

    def __init__(self, name, material, nx=0.0, ny=1.0, nz=0.0, d=0.0):
        super().__init__(name, material)
        target = gm.vec3_normalize(gm.vec3(nx, ny, nz))
        self.position = gm.f32([float(t) * d for t in target])
        self.rotation = gm.quat_rotation_to(gm.vec3(0, 1, 0), target)
        self.update_matrix()

    def get_orientation(self):
        n = gm.vec3_transform_quat(gm.vec3(0, 1, 0), self.rotation)
        return n, gm.vec3_dot(self.position, n)

    def schema(self):
        n, d = self.get_orientation()
        return [("vec3f", n), ("f32", d), ("i32", self.material._index)]


# ----------------------------------------------------------------------------- meshes
class ModelData:
    """tracer.js:912-1343: indexed triangle mesh; generate_bvh builds the BLAS natively."""

    def __init__(self, name="New Model", positions=None, normals=None, uvs=None, indices=None):
        self.name = name
        self.vertex_positions = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1)
        self.vertex_normals = np.ascontiguousarray(normals, dtype=np.float32).reshape(-1)
        self.vertex_texcoords = np.ascontiguousarray(uvs, dtype=np.float32).reshape(-1)
        self.index_positions = np.ascontiguousarray(indices, dtype=np.int64).reshape(-1)
        self.index_normals = self.index_positions
        self.index_texcoords = self.index_positions
        self.nodes: np.ndarray | None = None       # wgpt_bvh_node records (uint8 view of 32 B each)
        self.flat_triangles: np.ndarray | None = None
        self._node_offset = 0
        self._tri_offset = 0

    @classmethod
    def from_obj(cls, text, name: str = "New Model") -> "ModelData":
        """Model.parseOBJ + generateTriangles (tracer.js:949-1021) of an OBJ file's text, parsed
        natively (wgpt_parse_obj) with the reference's JavaScript number semantics."""
        raw = text.encode() if isinstance(text, str) else bytes(text)
        buf = np.frombuffer(raw, np.uint8) if raw else np.zeros(1, np.uint8)
        L = lib()
        nt, npos = C.c_uint32(0), C.c_uint32(0)
        check(L.wgpt_parse_obj(ptr(buf), len(raw), None, 0, C.byref(nt), None, 0, C.byref(npos)), "parse_obj")
        tris = np.zeros((nt.value, 24), np.float32)
        pos = np.zeros(npos.value, np.float32)
        check(L.wgpt_parse_obj(ptr(buf), len(raw), ptr(tris), nt.value, C.byref(nt), ptr(pos), npos.value,
                               C.byref(npos)), "parse_obj")
        m = cls(name, pos, np.zeros(0, np.float32), np.zeros(0, np.float32), np.zeros(0, np.int64))
        m._tris24 = tris
        return m

    def triangles24(self) -> np.ndarray:
        """generateTriangles (tracer.js:989-1021) as n x 24 float32 (v0 v1 v2 n0 n1 n2 uv0 uv1 uv2)."""
        if getattr(self, "_tris24", None) is not None:
            return self._tris24
        ip = self.index_positions.reshape(-1, 3)
        inn = self.index_normals.reshape(-1, 3)
        iuv = self.index_texcoords.reshape(-1, 3)
        P = self.vertex_positions.reshape(-1, 3)
        N = self.vertex_normals.reshape(-1, 3)
        U = self.vertex_texcoords.reshape(-1, 2)
        out = np.concatenate([P[ip[:, 0]], P[ip[:, 1]], P[ip[:, 2]], N[inn[:, 0]], N[inn[:, 1]], N[inn[:, 2]],
                              U[iuv[:, 0]], U[iuv[:, 1]], U[iuv[:, 2]]], axis=1)
        return np.ascontiguousarray(out, dtype=np.float32)

    def generate_bvh(self):
        t24 = self.triangles24()
        n = t24.shape[0]
        nodes = np.zeros((max(1, 2 * n - 1), 32), dtype=np.uint8)
        tris = np.zeros((n, 128), dtype=np.uint8)
        count = C.c_uint32(0)
        check(lib().wgpt_build_blas(ptr(t24), n, ptr(nodes), C.byref(count), ptr(tris)), "build_blas")
        self.nodes = nodes[: count.value].copy()
        self.flat_triangles = tris
        return self

    def root_bounds(self):
        f = self.nodes[0].view(np.float32)
        return f[0:3].copy(), f[4:7].copy()


class Model(Primitive):
    """tracer.js:1345-1417"""
    type = "Model"

    def __init__(self, name, material, model: ModelData, in_scene_bvh=True):
        super().__init__(name, material)
        self.model = model
        self.inSceneBVH = in_scene_bvh

    def get_bounds(self):
        world = gm.mat4_invert(self.invMatrix)
        pos = self.model.vertex_positions
        count = pos.size // 3
        if 0 < count < 5000:
            mn = gm.vec3(math.inf, math.inf, math.inf)
            mx = gm.vec3(-math.inf, -math.inf, -math.inf)
            for i in range(count):
                p = gm.vec3_transform_mat4(pos[i * 3:i * 3 + 3], world)
                mn = gm.vec3_min(mn, p)
                mx = gm.vec3_max(mx, p)
            return mn, mx
        lo, hi = self.model.root_bounds()
        return transform_aabb(lo, hi, world)

    def schema(self):
        return [("mat4x4f", self.invMatrix), ("i32", self.material._index), ("i32", self.lightIdx), ("i32", 0),
                ("u32", self.model._node_offset), ("vec3f", self.position), ("u32", self.model._tri_offset)]


# ----------------------------------------------------------------------------- camera, lights, scene
class Camera:
    """tracer.js:1419-1507"""

    def __init__(self, width: int, height: int):
        self.position = gm.vec3(0, 1.5, 4.5)
        self.target = gm.vec3(0, 0.5, 0)
        self.fov = 45.0
        self.aperture = 0.0
        self.focusDist = 1.0
        self.exposure = 1.0
        self.aspect = width / height
        self.ray00 = self.ray10 = self.ray01 = self.ray11 = gm.vec3()
        self.jitteredPosition = gm.vec3()

    def update_rays2(self, rand=None):
        """Corner rays at the focus plane; `rand` replaces Math.random for the lens sample."""
        sub = lambda a, b: gm.f32([float(a[i]) - float(b[i]) for i in range(3)])
        add = lambda a, b: gm.f32([float(a[i]) + float(b[i]) for i in range(3)])
        scale = lambda a, s: gm.f32([float(a[i]) * s for i in range(3)])
        sadd = lambda a, b, s: gm.f32([float(a[i]) + float(b[i]) * s for i in range(3)])
        look = sub(self.target, self.position)
        focus_dist = gm.vec3_length(look) * self.focusDist
        f = gm.vec3_normalize(look)
        r = gm.vec3_normalize(gm.vec3_cross(f, [0, 1, 0]))
        u = gm.vec3_cross(r, f)
        h = math.tan((self.fov * math.pi / 180) / 2) * focus_dist
        w = h * self.aspect
        hr = scale(r, w)
        hu = scale(u, h)
        fc = sadd(self.position, f, focus_dist)
        p00 = sub(sub(fc, hr), hu)
        p10 = sub(add(fc, hr), hu)
        p01 = add(sub(fc, hr), hu)
        p11 = add(add(fc, hr), hu)
        r1 = rand() if rand else 0.0
        r2 = rand() if rand else 0.0
        angle = r1 * math.pi * 2
        radius = math.sqrt(r2) * (self.aperture * 0.5)
        ox = math.cos(angle) * radius
        oy = math.sin(angle) * radius
        lens = sadd(gm.vec3(), r, ox)
        lens = sadd(lens, u, oy)
        self.jitteredPosition = add(self.position, lens)
        self.ray00 = sub(p00, self.jitteredPosition)
        self.ray10 = sub(p10, self.jitteredPosition)
        self.ray01 = sub(p01, self.jitteredPosition)
        self.ray11 = sub(p11, self.jitteredPosition)


class Light:
    """tracer.js:1692-1711"""

    def __init__(self, obj, index, area, power):
        self.obj = obj
        self.objIdx = index
        self.area = area
        self.power = power
        self.scale = 1.0
        if obj.type == "Sphere":
            avg = (float(obj.scale[0]) + float(obj.scale[1]) + float(obj.scale[2])) / 3
            obj.scale_set(avg, avg, avg)
            self.scale = avg
        elif obj.type == "Cube":
            self.scale = math.hypot(*[float(v) for v in obj.scale])

    def schema(self):
        return [("i32", self.objIdx), ("f32", self.area), ("f32", self.power), ("f32", self.scale),
                ("mat4x4f", self.obj.matrix)]


class Scene:
    """tracer.js:1621-1690"""

    def __init__(self, width: int, height: int):
        self.objects: list = []
        self.camera = Camera(width, height)
        self.bounces = 8
        self.background: HDRTexture | None = None

    def add(self, obj):
        self.objects.append(obj)
        return obj

    def get_materials(self):
        mats = []
        for o in self.objects:
            m = o.material
            if all(m is not x for x in mats):
                mats.append(m)
        return mats

    def get_textures(self):
        """tracer.js:1643-1653: distinct textures in material order, slot order within one."""
        texs = []
        for m in self.get_materials():
            for slot in TEXTURE_SLOTS:
                t = getattr(m, slot, None)
                if t is not None and all(t is not x for x in texs):
                    texs.append(t)
        return texs

    @staticmethod
    def light_power(obj):
        if obj.type not in ("Sphere", "Cube"):
            return 0.0, None
        m = obj.material
        if getattr(m, "emissiveTex", None) is not None:
            return 0.0, None
        lum = (0.2126 * m.emittance[0] + 0.7152 * m.emittance[1] + 0.0722 * m.emittance[2]) * m.emissionIntensity
        if lum <= 0:
            return 0.0, None
        area = obj.get_area()
        power = lum * area
        if power < 0.01:
            return 0.0, None
        return power, area

    def get_lights(self, objects):
        lights = []
        for i, o in enumerate(objects):
            if not o.enableNEE:
                continue
            power, area = self.light_power(o)
            if power <= 0:
                continue
            o.lightIdx = len(lights)
            lights.append(Light(o, i, area, power))
        return lights


# ----------------------------------------------------------------------------- packing
def pack_data_from_schema(objects, schema_of, empty_schema) -> tuple[np.ndarray, int]:
    """Renderer.packDataFromSchema (tracer.js:1772-1817) -> (uint8 buffer, stride)."""
    sample = schema_of(objects[0]) if objects else empty_schema
    stride = sum(4 if t == "pad" else SIZES[t] for t, _ in sample)
    stride = (stride + 15) & ~15
    count = max(1, len(objects))
    buf = bytearray(count * stride)
    for k, o in enumerate(objects):
        off = k * stride
        for t, d in schema_of(o):
            if t == "pad":
                off += 4
                continue
            if t in ("f32",):
                struct.pack_into("<f", buf, off, float(np.float32(d)))
            elif t == "i32":
                struct.pack_into("<i", buf, off, int(d))
            elif t == "u32":
                struct.pack_into("<I", buf, off, int(d) & 0xFFFFFFFF)
            else:
                arr = np.asarray(d, dtype=np.float64).astype(np.float32).reshape(-1)
                buf[off:off + 4 * arr.size] = arr.tobytes()
            off += SIZES[t]
    return np.frombuffer(bytes(buf), dtype=np.uint8).copy(), stride


_MAT_EMPTY = Material("name", [1, 1, 1], 1.0).schema()
_OBJ_EMPTY = [("mat4x4f", None), ("i32", 0), ("i32", 0), ("i32", 0), ("pad", None), ("vec3f", None), ("pad", None)]
_PLANE_EMPTY = [("vec3f", None), ("f32", 0), ("i32", 0)]
_MODEL_EMPTY = [("mat4x4f", None), ("i32", 0), ("i32", 0), ("i32", 0), ("u32", 0), ("vec3f", None), ("u32", 0)]
_LIGHT_EMPTY = [("i32", 0), ("f32", 0), ("f32", 0), ("f32", 0), ("mat4x4f", None)]


@dataclass
class PackedScene:
    """Byte buffers and pipeline constants of one scene (the WGSL bind group contents)."""
    materials: np.ndarray
    objects: np.ndarray
    tlas: np.ndarray
    meshes: np.ndarray
    bvh: np.ndarray
    triangles: np.ndarray
    planes: np.ndarray
    lights: np.ndarray
    sky_cdf: np.ndarray
    sky: np.ndarray
    sky_width: int
    sky_height: int
    sky_cdf_index: int
    sky_total_lum: float
    total_light_power: float
    bounce_limit: int
    flags: int
    textures: np.ndarray | None = None     # (layers, H, W, 4) uint8 texture array, or None
    sky_alias: np.ndarray | None = None    # (W*H, 2) uint32 alias table of the sky, or None
    extra: dict = field(default_factory=dict)


def build_tlas(objects) -> np.ndarray:
    """SceneBVHBuilder.rebuild + flatten over getBounds() of every object."""
    if not objects:
        return np.zeros(0, dtype=np.uint8)
    aabbs = np.zeros((len(objects), 6), dtype=np.float32)
    for i, o in enumerate(objects):
        lo, hi = o.get_bounds()
        aabbs[i, :3] = lo
        aabbs[i, 3:] = hi
    nodes = np.zeros((2 * len(objects) - 1, 32), dtype=np.uint8)
    count = C.c_uint32(0)
    check(lib().wgpt_build_tlas(ptr(aabbs), len(objects), ptr(nodes), C.byref(count)), "build_tlas")
    return nodes[: count.value].reshape(-1).copy()


def pack_scene_data(scene: Scene, prepare_textures: bool = True) -> PackedScene:
    """Renderer.packSceneData(true) (tracer.js:1819-1917) plus the sky texture and CDF of
    setScene (tracer.js:1976-2004).  With prepare_textures false (the updateObjects path,
    tracer.js:2136) the texture layers keep the texIndex values of the last full preparation,
    a texture that never had one packs as -1, and no texture array is built."""
    # prepareTextureArray runs first in setScene (tracer.js:1964): layers follow getTextures order
    textures = scene.get_textures() if prepare_textures else []
    for i, t in enumerate(textures):
        t.texIndex = i
    tex_array = None
    if textures:
        shape = textures[0].image.shape
        if any(t.image.shape != shape for t in textures):
            raise ValueError("every texture must have the array's common size (the reference resizes to 512 x 512)")
        tex_array = np.ascontiguousarray(np.stack([t.image for t in textures]), dtype=np.uint8)
    mats = scene.get_materials()
    has_height_maps = False
    for i, m in enumerate(mats):
        m._index = i
        if getattr(m, "heightTex", None) is not None:
            has_height_maps = True
    mat_buf, _ = pack_data_from_schema(mats, lambda m: m.schema(), _MAT_EMPTY)
    models = [o for o in scene.objects if o.type == "Model"]
    prims = [o for o in scene.objects if o.type in ("Sphere", "Cube", "Cylinder", "Torus")]
    in_bvh = [o for o in models if o.inSceneBVH]
    listed = [o for o in models if not o.inSceneBVH]
    planes = [o for o in scene.objects if o.type == "Plane"]
    scene_objects = prims + in_bvh
    for o in scene_objects:
        o.lightIdx = -1
    lights = scene.get_lights(scene_objects)
    light_buf, _ = pack_data_from_schema(lights, lambda l: l.schema(), _LIGHT_EMPTY)
    total_light_power = float(sum(l.power for l in lights))
    unique = []
    for o in models:
        if all(o.model is not u for u in unique):
            unique.append(o.model)
    n_nodes = n_tris = 0
    for m in unique:
        m._node_offset = n_nodes
        m._tri_offset = n_tris
        n_nodes += len(m.nodes)
        n_tris += len(m.flat_triangles)
    bvh = np.zeros(max(1, n_nodes) * 32, dtype=np.uint8)
    tris = np.zeros(max(1, n_tris) * 128, dtype=np.uint8)
    for m in unique:
        bvh[m._node_offset * 32:(m._node_offset + len(m.nodes)) * 32] = m.nodes.reshape(-1)
        tris[m._tri_offset * 128:(m._tri_offset + len(m.flat_triangles)) * 128] = m.flat_triangles.reshape(-1)
    tlas = build_tlas(scene_objects)
    obj_buf, _ = pack_data_from_schema(scene_objects, lambda o: o.schema(), _OBJ_EMPTY)
    plane_buf, _ = pack_data_from_schema(planes, lambda p: p.schema(), _PLANE_EMPTY)
    mesh_buf, _ = pack_data_from_schema(listed, lambda o: o.schema(), _MODEL_EMPTY)
    bg = scene.background if scene.background is not None else HDRTexture()
    cdf, cdf_index, total = bg.build_hdr_cdf()
    flags = 0
    flags |= HAS_SPHERES if any(o.type == "Sphere" for o in prims) else 0
    flags |= HAS_CUBES if any(o.type == "Cube" for o in prims) else 0
    flags |= HAS_CYLINDERS if any(o.type == "Cylinder" for o in prims) else 0
    flags |= HAS_TORI if any(o.type == "Torus" for o in prims) else 0
    flags |= HAS_MESHES if in_bvh else 0
    flags |= HAS_LIST_MESHES if listed else 0
    flags |= HAS_PLANES if planes else 0
    flags |= HAS_LIGHTS if lights else 0
    flags |= HAS_HEIGHTMAPS if has_height_maps else 0
    flags |= HAS_SKYBOX if scene.background is not None else 0
    flags |= MIS_SKYBOX if (scene.background is not None and not bg.plainColor and bg.enableNEE) else 0
    return PackedScene(
        materials=mat_buf, objects=obj_buf, tlas=tlas if tlas.size else np.zeros(32, dtype=np.uint8),
        meshes=mesh_buf, bvh=bvh, triangles=tris, planes=plane_buf, lights=light_buf, sky_cdf=cdf,
        sky=np.ascontiguousarray(bg.data, dtype=np.uint16), sky_width=bg.width, sky_height=bg.height,
        sky_cdf_index=cdf_index, sky_total_lum=total, total_light_power=total_light_power,
        bounce_limit=scene.bounces, flags=flags, textures=tex_array,
    )


def pack_params(scene: Scene, packed: PackedScene, width: int, height: int, frame: int, seed: int,
                section=(0, 0)) -> np.ndarray:
    """Renderer.updateUniforms (tracer.js:2207-2240) -> the 112-byte SceneParams."""
    cam = scene.camera
    b = bytearray(112)
    f = lambda off, v: struct.pack_into("<f", b, off, float(np.float32(v)))
    u = lambda off, v: struct.pack_into("<I", b, off, int(v) & 0xFFFFFFFF)
    for i in range(3):
        f(0 + 4 * i, cam.jitteredPosition[i])
        f(16 + 4 * i, cam.ray00[i])
        f(32 + 4 * i, cam.ray10[i])
        f(48 + 4 * i, cam.ray01[i])
        f(64 + 4 * i, cam.ray11[i])
    u(12, frame)
    u(28, width)
    u(44, height)
    f(60, cam.exposure)
    u(76, seed)
    u(80, packed.sky_width)
    u(84, packed.sky_height)
    f(88, packed.sky_total_lum)
    f(92, packed.total_light_power)
    u(96, section[0])
    u(100, section[1])
    u(104, packed.sky_cdf_index)
    return np.frombuffer(bytes(b), dtype=np.uint8).copy()
