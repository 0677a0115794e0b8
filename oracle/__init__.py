"""ORACLE -- test infrastructure only.

CPU restatement of the reference's shaders (pt_oracle.cpp, built into _build/liboracle.so) and of
its host-side builders (host_oracle.py).  Only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg use it, as the checker; the library in webgpuraytracer_b200/ never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboracle.so"

_P = C.c_void_p
_U32 = C.c_uint32
_lib = None


def build(force: bool = False) -> Path:
    """Compiles liboracle.so with the Makefile next to this file."""
    cmd = ["make", "-C", str(HERE)] + (["-B"] if force else [])
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")
    return LIB_PATH


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = C.CDLL(str(LIB_PATH))
        L.oracle_render.argtypes = [_P, _P, _P, _P, _U32, _U32, _U32, _U32, _U32, _U32, _P, _P, C.c_int, _P]
        L.oracle_gbuffer.argtypes = [_P, _P, _P, _P, _U32, _U32, _U32, _U32, _P, _P, C.c_int]
        L.oracle_trace_closest.argtypes = [_P, _P, _P, _P, _U32, _P, _P, _P, _P, _P, C.c_int]
        L.oracle_bsdf.argtypes = [_P, _P, C.c_float, C.c_float, _P, _P, _U32, _P, _P]
        L.oracle_rng_stream.argtypes = [_U32, _U32, _U32, _U32, _P]
        L.oracle_denoise.argtypes = [_P, _P, _P, _P, _U32, _P, _P, _P, C.c_int]
        L.oracle_resample.argtypes = [_P, _U32, _U32, _P, _U32, _U32, C.c_float, C.c_float]
        L.oracle_builtin.argtypes = [C.c_int, _P, _P, _U32, _P]
        L.oracle_sample_texture.argtypes = [_P, _U32, _U32, _U32, C.c_int32, _P, _U32, _P]
        L.oracle_sample_texture.restype = None
        L.oracle_render_f64.argtypes = [_P, _P, _P, _P, _U32, _U32, _U32, _U32, _U32, _U32, _P, C.c_int]
        L.oracle_render_f64.restype = C.c_int
        L.oracle_sample_env.argtypes = [_P, _P, _P, _P, _P, _U32, _P, _P]
        L.oracle_sample_env.restype = C.c_int
        L.oracle_sample_surface.argtypes = [_P, _P, C.c_float, C.c_float, _P, _P, _U32, _P, _P]
        L.oracle_sample_surface.restype = C.c_int
        for name in ("oracle_render", "oracle_gbuffer", "oracle_trace_closest", "oracle_bsdf", "oracle_denoise",
                     "oracle_resample"):
            getattr(L, name).restype = C.c_int
        L.oracle_rng_stream.restype = None
        L.oracle_builtin.restype = None
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


class OracleScene:
    """Pointers of one packed scene in the order pt_oracle.cpp expects."""

    def __init__(self, packed):
        self.packed = packed
        tex = packed.textures if packed.textures is not None else np.zeros((1, 1, 1, 4), np.uint8)
        bufs = [packed.materials, packed.objects, packed.tlas, packed.meshes, packed.bvh, packed.triangles,
                packed.planes, packed.lights, packed.sky_cdf, packed.sky, tex]
        self._keep = [np.ascontiguousarray(b) for b in bufs]
        self.ptrs = (C.c_void_p * 11)(*[b.ctypes.data for b in self._keep])
        self.sizes = np.array([b.nbytes for b in self._keep], dtype=np.uint64)
        layers = tex.shape[0] if packed.textures is not None else 0
        self.meta = np.array([packed.sky_width, packed.sky_height, packed.bounce_limit, packed.flags,
                              tex.shape[2], tex.shape[1], layers], dtype=np.uint32)

    def args(self):
        return (C.cast(self.ptrs, C.c_void_p), _p(self.sizes), _p(self.meta))


def render(oscene: OracleScene, params: np.ndarray, first_frame: int, reps: int, section, accum: np.ndarray,
           out: np.ndarray, nthreads: int = 0, counters: np.ndarray | None = None) -> int:
    sx, sy, sw, sh = section
    return lib().oracle_render(*oscene.args(), _p(params), first_frame, reps, sx, sy, sw, sh, _p(accum), _p(out),
                               nthreads, _p(counters))


def render_f64(oscene: OracleScene, params: np.ndarray, first_frame: int, reps: int, section,
               acc8: np.ndarray, nthreads: int = 0) -> int:
    """oracle_render with FP64 Welford accumulation into acc8 (H, W, 8) float64 (zeroed first)."""
    sx, sy, sw, sh = section
    assert acc8.dtype == np.float64 and acc8.flags.c_contiguous
    return lib().oracle_render_f64(*oscene.args(), _p(params), first_frame, reps, sx, sy, sw, sh, _p(acc8), nthreads)


def gbuffer(oscene: OracleScene, params: np.ndarray, section, gbuf: np.ndarray, out: np.ndarray,
            nthreads: int = 0) -> int:
    sx, sy, sw, sh = section
    return lib().oracle_gbuffer(*oscene.args(), _p(params), sx, sy, sw, sh, _p(gbuf), _p(out), nthreads)


def trace_closest(oscene: OracleScene, rays: np.ndarray, nthreads: int = 0):
    rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 6)
    n = rays.shape[0]
    o = np.empty(n, np.int32)
    m = np.empty(n, np.int32)
    pr = np.empty(n, np.int32)
    t = np.empty(n, np.float32)
    nn = np.empty((n, 3), np.float32)
    lib().oracle_trace_closest(*oscene.args(), _p(rays), n, _p(o), _p(m), _p(pr), _p(t), _p(nn), nthreads)
    return o, m, pr, t, nn


def sample_env(oscene: OracleScene, params: np.ndarray, u2: np.ndarray):
    """sample_env_cdf of each random pair: (texel (n, 2) as x, y; pdf (n,))."""
    u2 = np.ascontiguousarray(u2, np.float32).reshape(-1, 2)
    n = u2.shape[0]
    texel = np.empty((n, 2), np.uint32)
    pdf = np.empty(n, np.float32)
    lib().oracle_sample_env(*oscene.args(), _p(params), _p(u2), n, _p(texel), _p(pdf))
    return texel, pdf


def sample_surface(material144: np.ndarray, normal, roughness, metallic, albedo, V, rng_state: int):
    """One sample_surface call in air: (continues, new direction (3,), throughput (3,))."""
    d = np.empty(3, np.float32)
    tp = np.empty(3, np.float32)
    nrm = np.asarray(normal, np.float32)
    alb = np.asarray(albedo, np.float32)
    v = np.asarray(V, np.float32)
    cont = lib().oracle_sample_surface(_p(material144), _p(nrm), roughness, metallic, _p(alb), _p(v),
                                       rng_state & 0xFFFFFFFF, _p(d), _p(tp))
    return bool(cont), d, tp


def rng_stream(idx: int, sample_number: int, seed: int, n: int) -> np.ndarray:
    out = np.empty(n, np.float32)
    lib().oracle_rng_stream(idx, sample_number, seed, n, _p(out))
    return out


def denoise(color: np.ndarray, gbuf: np.ndarray, uniforms: np.ndarray, steps: np.ndarray, nthreads: int = 0):
    h, w = color.shape[:2]
    filt = np.empty((h, w, 4), np.float32)
    comp = np.empty((h, w, 4), np.float32)
    out = np.empty((h, w, 4), np.uint8)
    steps = np.ascontiguousarray(steps, dtype=np.uint32)
    lib().oracle_denoise(_p(np.ascontiguousarray(color, np.float32)), _p(np.ascontiguousarray(gbuf, np.float32)),
                         _p(uniforms), _p(steps), len(steps), _p(filt), _p(comp), _p(out), nthreads)
    return filt, comp, out


def resample(src: np.ndarray, dst_w: int, dst_h: int, rx: float, ry: float) -> np.ndarray:
    h, w = src.shape[:2]
    dst = np.empty((dst_h, dst_w, 4), np.uint8)
    lib().oracle_resample(_p(np.ascontiguousarray(src, np.uint8)), w, h, _p(dst), dst_w, dst_h, rx, ry)
    return dst


def bsdf(material144: np.ndarray, normal, roughness, metallic, albedo, vl: np.ndarray):
    vl = np.ascontiguousarray(vl, np.float32).reshape(-1, 6)
    n = vl.shape[0]
    f = np.empty((n, 3), np.float32)
    pdf = np.empty(n, np.float32)
    nrm = np.asarray(normal, np.float32)
    alb = np.asarray(albedo, np.float32)
    lib().oracle_bsdf(_p(material144), _p(nrm), roughness, metallic, _p(alb), _p(vl), n, _p(f), _p(pdf))
    return f, pdf


def builtin(op: int, x: np.ndarray, y: np.ndarray | None = None) -> np.ndarray:
    x = np.ascontiguousarray(x, np.float32)
    y = np.zeros_like(x) if y is None else np.ascontiguousarray(y, np.float32)
    out = np.empty_like(x)
    lib().oracle_builtin(op, _p(x), _p(y), x.size, _p(out))
    return out


def sample_texture(textures: np.ndarray, layer: int, uv: np.ndarray) -> np.ndarray:
    """The material sampler on a (layers, H, W, 4) uint8 array at uv (n, 2); returns (n, 4) float32."""
    tex = np.ascontiguousarray(textures, np.uint8)
    uv = np.ascontiguousarray(uv, np.float32).reshape(-1, 2)
    out = np.empty((uv.shape[0], 4), np.float32)
    lib().oracle_sample_texture(_p(tex), tex.shape[2], tex.shape[1], tex.shape[0], layer, _p(uv), uv.shape[0], _p(out))
    return out


def default_threads() -> int:
    return os.cpu_count() or 1
