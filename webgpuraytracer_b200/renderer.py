"""Renderer and Denoiser over libwgpt.so, mirroring tracer.js's classes of the same names.

    Renderer.set_scene      setScene       (tracer.js:1955-2102)
    Renderer.update_objects updateObjects  (tracer.js:2132-2164)
    Renderer.resize         resize         (tracer.js:2166-2205)
    Renderer.update_uniforms updateUniforms (tracer.js:2207-2240)
    Renderer.render         render         (tracer.js:2242-2297), tile by tile
    Renderer.render_preview renderPreview  (tracer.js:2334-2392), with the scale.wgsl blit
    Denoiser.execute        execute        (tracer.js:2583-2637)

Device work goes through the C ABI only; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import scene as sc
from ._lib import ENV_ALIAS, ENV_CDF, SceneDesc, Buffer, WavefrontTuning, check, lib, ptr


def _buf(a: np.ndarray | None) -> Buffer:
    if a is None or a.size == 0:
        return Buffer(None, 0)
    return Buffer(ptr(a), a.nbytes)


def scene_desc(p: sc.PackedScene) -> SceneDesc:
    d = SceneDesc()
    d.materials = _buf(p.materials)
    d.objects = _buf(p.objects)
    d.tlas = _buf(p.tlas)
    d.meshes = _buf(p.meshes)
    d.bvh = _buf(p.bvh)
    d.triangles = _buf(p.triangles)
    d.planes = _buf(p.planes)
    d.lights = _buf(p.lights)
    d.sky_cdf = _buf(p.sky_cdf)
    d.sky_rgba16f = ptr(p.sky)
    d.sky_width = p.sky_width
    d.sky_height = p.sky_height
    d.bounce_limit = p.bounce_limit
    d.feature_flags = p.flags
    if p.textures is not None:
        d.textures_rgba8 = ptr(p.textures)
        d.tex_layers, d.tex_height, d.tex_width = p.textures.shape[:3]
    if p.sky_alias is not None:
        d.sky_alias = ptr(p.sky_alias)
    return d


class Renderer:
    def __init__(self, width: int, height: int, device: int = 0, seed_fn=None):
        self.width, self.height = int(width), int(height)
        self.L = lib()
        h = C.c_void_p()
        check(self.L.wgpt_create(device, C.byref(h)), "wgpt_create")
        self.ctx = h
        self.scene: sc.Scene | None = None
        self.packed: sc.PackedScene | None = None
        self.frame = 0
        self.isgbuf = False
        # the reference draws a fresh Math.random() seed per dispatch; tests pin it
        self.seed_fn = seed_fn or (lambda: 1)
        self.section = (0, 0, self.width, self.height)

    # -- lifetime
    def close(self):
        if self.ctx:
            self.L.wgpt_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        check(rc, what, self.ctx)

    # -- scene
    def set_scene(self, scene: sc.Scene, isgbuf: bool = False, packed: sc.PackedScene | None = None):
        self.scene = scene
        self.isgbuf = isgbuf
        self.packed = packed if packed is not None else sc.pack_scene_data(scene)
        self._desc = scene_desc(self.packed)
        self._check(self.L.wgpt_upload_scene(self.ctx, C.byref(self._desc)), "upload_scene")
        self.resize()

    def update_objects(self, packed: sc.PackedScene | None = None) -> bool:
        """Renderer.updateObjects (tracer.js:2132-2164): repacks the scene and rewrites objects,
        TLAS, planes, list meshes and materials in place when the flags match and everything
        fits (lights, BLAS, sky and textures stay as uploaded, as in the reference); otherwise a
        full set_scene.  Returns True when the fast path was taken."""
        packed = packed if packed is not None else sc.pack_scene_data(self.scene, prepare_textures=False)
        if packed.sky_alias is None and self.packed is not None:
            packed.sky_alias = self.packed.sky_alias     # the sky is not rewritten either
        desc = scene_desc(packed)
        rc = self.L.wgpt_update_objects(self.ctx, C.byref(desc))
        if rc == 7:   # WGPT_E_REBUILD: SLOW PATH, full scene rebuild (setScene prepares the textures)
            self.set_scene(self.scene, self.isgbuf)
            return False
        self._check(rc, "update_objects")
        # the uniforms take the new total light power (tracer.js:1841, 2234) while the light buffer stays
        self.packed, self._desc = packed, desc
        return True

    def resize(self, width: int | None = None, height: int | None = None):
        if width is not None:
            self.width, self.height = int(width), int(height)
        self._check(self.L.wgpt_resize(self.ctx, self.width, self.height, 1 if self.isgbuf else 0), "resize")
        self.reset()

    def reset(self):
        self.frame = 0

    # -- dispatch
    def update_uniforms(self, frame: int | None = None, section=(0, 0)):
        cam = self.scene.camera
        cam.update_rays2()
        params = sc.pack_params(self.scene, self.packed, self.width, self.height,
                                self.frame if frame is None else frame, self.seed_fn(), section)
        self._params = params
        self._check(self.L.wgpt_set_params(self.ctx, ptr(params)), "set_params")
        return params

    def render_section(self, first_frame: int, reps: int, x: int, y: int, w: int, h: int):
        self.update_uniforms(first_frame, (x, y))
        self._check(self.L.wgpt_render(self.ctx, first_frame, reps, x, y, w, h), "render")

    def render(self, tsize: int = 256, reps: int = 1, sync: bool = True):
        """Tiled progressive render: every tile gets `reps` samples (frames frame..frame+reps-1)."""
        start = self.frame
        tiles_x = math.ceil(self.width / tsize)
        tiles_y = math.ceil(self.height / tsize)
        for ty in range(tiles_y):
            for tx in range(tiles_x):
                left, top = tx * tsize, ty * tsize
                w = min(tsize, self.width - left)
                h = min(tsize, self.height - top)
                self.section = (left, top, w, h)
                self.render_section(start, reps, left, top, w, h)
        if sync:
            self.synchronize()
        self.frame = start + reps

    def render_gbuffer(self):
        self.update_uniforms(self.frame, (0, 0))
        self._check(self.L.wgpt_render_gbuffer(self.ctx, 0, 0, self.width, self.height), "render_gbuffer")
        self.synchronize()

    def render_preview(self, preview_size: float) -> np.ndarray:
        """renderPreview (tracer.js:2334-2392) at a given preview size: one sample of the reduced
        pWidth x pHeight image into the canvas-sized buffers, then the scale.wgsl blit to the
        canvas.  Returns the canvas image (rgba8)."""
        cw, ch = self.width, self.height
        maxsize = math.floor(preview_size)
        scale = min(maxsize / cw, maxsize / ch)
        pw, ph = int(math.floor(cw * scale)), int(math.floor(ch * scale))
        self.scene.camera.update_rays2()
        params = sc.pack_params(self.scene, self.packed, pw, ph, self.frame, self.seed_fn(), (0, 0))
        self._params = params
        self._check(self.L.wgpt_set_params(self.ctx, ptr(params)), "set_params")
        self._check(self.L.wgpt_render(self.ctx, self.frame, 1, 0, 0, pw, ph), "render")
        rx = float(np.float32(pw / cw))
        ry = float(np.float32(ph / ch))
        canvas = self.resample(cw, ch, rx, ry)
        self.frame += 1
        return canvas

    def synchronize(self):
        self._check(self.L.wgpt_synchronize(self.ctx), "synchronize")

    def wait(self, timeout_ms: int) -> bool:
        """Host watchdog: True once the queued work finished, False if it is still running after
        timeout_ms (it keeps running); kernel-reported errors raise as in synchronize()."""
        rc = self.L.wgpt_synchronize_timeout(self.ctx, int(timeout_ms))
        if rc == 10:   # WGPT_E_TIMEOUT
            return False
        self._check(rc, "synchronize_timeout")
        return True

    # -- checkpoint / resume (long converged renders)
    def save_state(self, path):
        """Writes the accumulation (FP32 running mean, and the FP64 Welford records when they are
        on), the frame count and the image size to an .npz file."""
        state = {"accum": self.read_accum(), "frame": np.int64(self.frame),
                 "size": np.array([self.width, self.height], np.int64)}
        if getattr(self, "_acc64_on", False):
            a = np.empty((self.height, self.width, 8), np.float64)
            self._check(self.L.wgpt_read_accum_f64(self.ctx, ptr(a)), "read_accum_f64")
            state["accum64"] = a
        np.savez(path, **state)

    def load_state(self, path):
        """Restores a save_state() file into this renderer (same image size; the FP64 records
        are restored when the file has them, switching FP64 accumulation on)."""
        with np.load(path) as f:
            w, h = (int(v) for v in f["size"])
            if (w, h) != (self.width, self.height):
                raise ValueError(f"checkpoint is {w}x{h}, renderer is {self.width}x{self.height}")
            self.write_accum(np.ascontiguousarray(f["accum"], np.float32))
            if "accum64" in f.files:
                self.set_accum_f64(True)
                a = np.ascontiguousarray(f["accum64"], np.float64)
                self._check(self.L.wgpt_write_accum_f64(self.ctx, ptr(a)), "write_accum_f64")
            self.frame = int(f["frame"])

    # -- readback
    def read_accum(self) -> np.ndarray:
        a = np.empty((self.height, self.width, 4), dtype=np.float32)
        self._check(self.L.wgpt_read_accum(self.ctx, ptr(a)), "read_accum")
        return a

    def write_accum(self, a: np.ndarray):
        a = np.ascontiguousarray(a, dtype=np.float32)
        self._check(self.L.wgpt_write_accum(self.ctx, ptr(a)), "write_accum")

    def read_output(self) -> np.ndarray:
        a = np.empty((self.height, self.width, 4), dtype=np.uint8)
        self._check(self.L.wgpt_read_output(self.ctx, ptr(a)), "read_output")
        return a

    def read_gbuffer(self) -> np.ndarray:
        a = np.empty((self.height, self.width, 12), dtype=np.float32)
        self._check(self.L.wgpt_read_gbuffer(self.ctx, ptr(a)), "read_gbuffer")
        return a

    def write_gbuffer(self, g: np.ndarray):
        g = np.ascontiguousarray(g, dtype=np.float32)
        self._check(self.L.wgpt_write_gbuffer(self.ctx, ptr(g)), "write_gbuffer")

    def trace_rays(self, rays: np.ndarray):
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 6)
        n = rays.shape[0]
        o = np.empty(n, np.int32)
        m = np.empty(n, np.int32)
        p = np.empty(n, np.int32)
        t = np.empty(n, np.float32)
        nn = np.empty((n, 3), np.float32)
        self._check(self.L.wgpt_trace_rays(self.ctx, ptr(rays), n, ptr(o), ptr(m), ptr(p), ptr(t), ptr(nn)),
                    "trace_rays")
        return o, m, p, t, nn

    def set_accum_f64(self, on: bool = True):
        """FP64 Welford accumulation of every sample next to the FP32 running mean."""
        self._check(self.L.wgpt_set_accum_f64(self.ctx, 1 if on else 0), "set_accum_f64")
        self._acc64_on = bool(on)

    def read_accum_f64(self):
        """(mean (H, W, 3), per-sample variance (H, W, 3), sample count (H, W)) in float64."""
        a = np.empty((self.height, self.width, 8), np.float64)
        self._check(self.L.wgpt_read_accum_f64(self.ctx, ptr(a)), "read_accum_f64")
        n = a[..., 6]
        var = a[..., 3:6] / np.maximum(n - 1.0, 1.0)[..., None]
        return a[..., 0:3], var, n

    def set_render_mode(self, mode: int):
        """MODE_WAVEFRONT (path pool with regeneration) or MODE_MEGAKERNEL (one thread per pixel)."""
        self._check(self.L.wgpt_set_render_mode(self.ctx, int(mode)), "set_render_mode")

    def set_env_sampling(self, mode: int):
        """ENV_CDF (the reference's CDF search, bit-exact) or ENV_ALIAS (O(1) alias table, same
        texel probabilities: statistically equal images).  ENV_ALIAS builds the sky's alias table
        and uploads the scene again when the current upload has none (the frame count restarts)."""
        if mode == ENV_ALIAS and self.packed is not None and self.packed.sky_alias is None:
            self.packed.sky_alias = self.scene.background.build_env_alias()
            self.set_scene(self.scene, self.isgbuf, packed=self.packed)
        self._check(self.L.wgpt_set_env_sampling(self.ctx, int(mode)), "set_env_sampling")

    def set_wavefront_config(self, pool_paths: int = 0, units_per_pass: int = 0):
        """Path-slot pool size and samples per pass of the wavefront renderer (0 keeps a value)."""
        self._check(self.L.wgpt_set_wavefront_config(self.ctx, int(pool_paths), int(units_per_pass)),
                    "set_wavefront_config")

    def set_wavefront_tuning(self, trav_shape: int = 2, shade_block: int = 512, refill_closest: int = 24,
                             refill_shadow: int = 8, shadow_wide: int = 0):
        """Kernel variants and thresholds of the wavefront renderer (results do not depend on
        them): traversal block shape 0 (192 x 6), 1 (128 x 9) or 2 (256 x 4); surface-shading
        block 512 or 256; idle lanes a traversal warp gathers before refilling (1..32); shadow
        rays over the 4-wide view of the BVHs (1) or the 2-wide trees (0)."""
        t = WavefrontTuning(trav_shape, shade_block, refill_closest, refill_shadow, shadow_wide)
        self._check(self.L.wgpt_set_wavefront_tuning(self.ctx, C.byref(t)), "set_wavefront_tuning")

    def wavefront_tuning(self) -> dict:
        t = WavefrontTuning()
        self._check(self.L.wgpt_get_wavefront_tuning(self.ctx, C.byref(t)), "get_wavefront_tuning")
        return {"trav_shape": int(t.trav_shape), "shade_block": int(t.shade_block),
                "refill_closest": int(t.refill_closest), "refill_shadow": int(t.refill_shadow),
                "shadow_wide": int(t.shadow_wide)}

    def wavefront_config(self) -> tuple[int, int]:
        pool, units = C.c_uint32(0), C.c_uint64(0)
        self._check(self.L.wgpt_get_wavefront_config(self.ctx, C.byref(pool), C.byref(units)),
                    "get_wavefront_config")
        return int(pool.value), int(units.value)

    # -- batched views (many cameras of the uploaded scene in one call)
    def set_views(self, sizes):
        """Allocates one image pair (accumulation, rgba8) per (width, height)."""
        w = np.array([x[0] for x in sizes], np.uint32)
        h = np.array([x[1] for x in sizes], np.uint32)
        self._views = [(int(a), int(b)) for a, b in zip(w, h)]
        self._check(self.L.wgpt_set_views(self.ctx, len(w), ptr(w), ptr(h)), "set_views")

    def render_views(self, params, first_frames, spp, timing: bool = True):
        """Adds spp[i] samples to view i (params: n x 112-byte SceneParams).  Returns the
        per-view completion times in ms from the start of the call's work (timing=True)."""
        blob = np.ascontiguousarray(np.concatenate([np.frombuffer(np.asarray(p).tobytes(), np.uint8)
                                                    for p in params]))
        ff = np.ascontiguousarray(first_frames, np.uint32)
        sp = np.ascontiguousarray(spp, np.uint32)
        done = np.full(len(ff), -1.0, np.float32)
        self._check(self.L.wgpt_render_views(self.ctx, ptr(blob), ptr(ff), ptr(sp), ptr(done) if timing else None),
                    "render_views")
        return done

    def render_views_gbuffer(self, params):
        """gbuf_main for every view (allocates the view G-buffers on first use)."""
        blob = np.ascontiguousarray(np.concatenate([np.frombuffer(np.asarray(p).tobytes(), np.uint8)
                                                    for p in params]))
        self._check(self.L.wgpt_render_views_gbuffer(self.ctx, ptr(blob)), "render_views_gbuffer")

    def read_view(self, i: int):
        w, h = self._views[i]
        acc = np.empty((h, w, 4), np.float32)
        out = np.empty((h, w, 4), np.uint8)
        self._check(self.L.wgpt_read_view(self.ctx, i, ptr(acc), ptr(out)), "read_view")
        return acc, out

    def set_counting(self, on: bool):
        self._check(self.L.wgpt_set_counting(self.ctx, 1 if on else 0), "set_counting")

    def read_counters(self) -> np.ndarray:
        a = np.zeros(16, dtype=np.uint64)
        self._check(self.L.wgpt_read_counters(self.ctx, ptr(a)), "read_counters")
        return a

    def stream_handle(self) -> int:
        return int(self.L.wgpt_stream(self.ctx) or 0)

    def resample(self, dst_w: int, dst_h: int, rx: float, ry: float) -> np.ndarray:
        self._check(self.L.wgpt_resample(self.ctx, dst_w, dst_h, rx, ry), "resample")
        out = np.empty((dst_h, dst_w, 4), dtype=np.uint8)
        self._check(self.L.wgpt_read_canvas(self.ctx, ptr(out), dst_w, dst_h), "read_canvas")
        return out


def denoise_uniforms(width, height, passes=4, sigma_color=0.30, sigma_normal=128.0, sigma_depth=0.2,
                     sigma_albedo=0.07, sigma_material=0.07, glossy_protect=0.75, exposure=1.0,
                     use_median=True, use_demodulate=True, step_width=1) -> np.ndarray:
    """Denoiser.updateUniforms (tracer.js:2560-2581) with the constructor defaults (2424-2435)."""
    u = np.zeros(12, dtype=np.uint32)
    f = u.view(np.float32)
    u[0], u[1], u[2], u[3] = width, height, step_width, passes
    f[4], f[5], f[6], f[7], f[8], f[9], f[10] = (sigma_color, sigma_normal, sigma_depth, sigma_albedo,
                                                 sigma_material, glossy_protect, exposure)
    u[11] = (1 if use_median else 0) | (2 if use_demodulate else 0)
    return u.view(np.uint8).copy()


def step_schedule(passes: int, mode: str = "intended") -> np.ndarray:
    """Step widths per a-trous pass.  "intended": 1, 2, 4, ... (tracer.js:2603 computes 1 << i);
    "as_run": every pass sees 2^(passes-1), because all queue.writeBuffer calls land before the
    single submit (tracer.js:2605 + 2636)."""
    if mode == "intended":
        return np.array([1 << i for i in range(passes)], dtype=np.uint32)
    if mode == "as_run":
        return np.full(passes, 1 << (passes - 1) if passes else 1, dtype=np.uint32)
    raise ValueError(mode)


class Denoiser:
    """tracer.js:2418-2638"""

    def __init__(self, renderer: Renderer, passes: int = 4, mode: str = "intended", **params):
        self.r = renderer
        self.passes = passes
        self.mode = mode
        self.params = params
        self.exposure = renderer.scene.camera.exposure if renderer.scene else 1.0

    def execute(self):
        u = denoise_uniforms(self.r.width, self.r.height, self.passes, exposure=self.exposure, **self.params)
        steps = step_schedule(self.passes, self.mode)
        self.r._check(self.r.L.wgpt_denoise(self.r.ctx, ptr(u), ptr(steps), self.passes), "denoise")
        self.r.synchronize()

    def read(self):
        n = self.r.width * self.r.height
        filt = np.empty((self.r.height, self.r.width, 4), dtype=np.float32)
        comp = np.empty((self.r.height, self.r.width, 4), dtype=np.float32)
        self.r._check(self.r.L.wgpt_read_denoised(self.r.ctx, ptr(filt), ptr(comp)), "read_denoised")
        return filt, comp, self.r.read_output()
