"""Learned kernel-predicting denoiser (host side of wgpt_kpcn_*).

The network runs and trains on the GPU through the C ABI; this module holds its layer table
(mirroring kpcn.cu, for tools that read the flat parameter array), the training-example
generator that renders (noisy, G-buffer, target) triples with the path tracer itself, and the
image metrics used to compare it with the a-trous filter.
"""
from __future__ import annotations

import ctypes as C
import json
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import renderer as rd
from . import scene as sc
from ._lib import WgptError, lib, ptr


@dataclass(frozen=True)
class LayerSpec:
    name: str
    cu: int        # upsampled coarse input channels (padded)
    cs: int        # same-resolution input channels (padded)
    cout: int      # output channels (padded)
    taps: int      # 9 (3x3) or 1
    relu: bool
    level: int     # resolution level of the output (0 = full)

    @property
    def cin(self) -> int:
        return self.cu + self.cs

    @property
    def n_weights(self) -> int:
        return self.cout * self.taps * self.cin


LAYERS = (
    LayerSpec("E0a", 0, 16, 32, 9, True, 0),
    LayerSpec("E0", 0, 32, 32, 9, True, 0),
    LayerSpec("E1", 0, 32, 48, 9, True, 1),
    LayerSpec("E2", 0, 48, 64, 9, True, 2),
    LayerSpec("E3", 0, 64, 96, 9, True, 3),
    LayerSpec("E4a", 0, 96, 128, 9, True, 4),
    LayerSpec("E4", 0, 128, 128, 9, True, 4),
    LayerSpec("D3", 128, 96, 96, 9, True, 3),
    LayerSpec("D2", 96, 64, 64, 9, True, 2),
    LayerSpec("D1", 64, 48, 48, 9, True, 1),
    LayerSpec("D0", 48, 32, 32, 9, True, 0),
    LayerSpec("OUT", 0, 32, 80, 1, False, 0),
)


def param_slices() -> dict[str, tuple[slice, slice]]:
    """Per layer: (weights, bias) slices of the flat parameter array."""
    out, off = {}, 0
    for l in LAYERS:
        w = slice(off, off + l.n_weights)
        off += l.n_weights
        b = slice(off, off + l.cout)
        off += l.cout
        out[l.name] = (w, b)
    return out


N_PARAMS = sum(l.n_weights + l.cout for l in LAYERS)


class Kpcn:
    """wgpt_kpcn_* through ctypes."""

    def __init__(self, device: int = 0, seed: int = 1):
        self.L = lib()
        h = C.c_void_p()
        rc = self.L.wgpt_kpcn_create(device, seed, C.byref(h))
        if rc != 0:
            raise WgptError(rc, "wgpt_kpcn_create")
        self.h = h.value
        n = C.c_uint64()
        self._check(self.L.wgpt_kpcn_num_params(self.h, C.byref(n)), "num_params")
        self.n_params = int(n.value)

    def _check(self, rc: int, what: str):
        if rc != 0:
            msg = self.L.wgpt_kpcn_last_error(self.h) if getattr(self, "h", None) else b""
            raise WgptError(rc, what, (msg or b"").decode())

    def close(self):
        if getattr(self, "h", None):
            self.L.wgpt_kpcn_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get_params(self) -> np.ndarray:
        a = np.empty(self.n_params, np.float32)
        self._check(self.L.wgpt_kpcn_get_params(self.h, ptr(a)), "get_params")
        return a

    def set_params(self, a: np.ndarray):
        a = np.ascontiguousarray(a, np.float32)
        assert a.size == self.n_params
        self._check(self.L.wgpt_kpcn_set_params(self.h, ptr(a)), "set_params")

    def add_example(self, noisy: np.ndarray, gbuf: np.ndarray, target: np.ndarray):
        h, w = noisy.shape[:2]
        noisy = np.ascontiguousarray(noisy, np.float32)
        gbuf = np.ascontiguousarray(gbuf, np.float32)
        target = np.ascontiguousarray(target, np.float32)
        assert noisy.shape == (h, w, 4) and target.shape == (h, w, 4) and gbuf.shape == (h, w, 12)
        self._check(self.L.wgpt_kpcn_add_example(self.h, ptr(noisy), ptr(gbuf), ptr(target), w, h), "add_example")

    def train(self, steps: int, batch: int = 8, crop: int = 64, lr: float = 1e-3, seed: int = 1) -> np.ndarray:
        losses = np.zeros(steps, np.float32)
        self._check(self.L.wgpt_kpcn_train(self.h, steps, batch, crop, lr, seed, ptr(losses)), "train")
        return losses

    def grads(self, batch: int, crop: int, seed: int, dev_grads) -> float:
        """Forward and backward of `batch` crops drawn with `seed`; the FP32 gradient goes into
        dev_grads (a CUDA tensor of num_params floats on this denoiser's device).  Returns the
        batch loss."""
        loss = np.zeros(1, np.float32)
        self._check(self.L.wgpt_kpcn_grads(self.h, batch, crop, seed, ptr(loss), C.c_void_p(dev_grads.data_ptr())),
                    "grads")
        return float(loss[0])

    def apply(self, dev_grads, scale: float, lr: float):
        """One Adam step with the gradient dev_grads * scale."""
        self._check(self.L.wgpt_kpcn_apply(self.h, C.c_void_p(dev_grads.data_ptr()), scale, lr), "apply")

    def loss_and_grads(self, noisy, gbuf, target):
        h, w = noisy.shape[:2]
        noisy = np.ascontiguousarray(noisy, np.float32)
        gbuf = np.ascontiguousarray(gbuf, np.float32)
        target = np.ascontiguousarray(target, np.float32)
        loss = np.zeros(1, np.float32)
        grads = np.zeros(self.n_params, np.float32)
        out = np.zeros((h, w, 4), np.float32)
        self._check(self.L.wgpt_kpcn_loss_and_grads(self.h, ptr(noisy), ptr(gbuf), ptr(target), w, h, ptr(loss),
                                                    ptr(grads), ptr(out)), "loss_and_grads")
        return float(loss[0]), grads, out

    def denoise(self, r: rd.Renderer, exposure: float = 1.0, want_linear: bool = True):
        """Filters the renderer's accumulation with its G-buffer into its rgba8 image."""
        lin = np.zeros((r.height, r.width, 4), np.float32) if want_linear else None
        self._check(self.L.wgpt_kpcn_denoise(self.h, r.ctx, exposure, ptr(lin) if want_linear else None), "denoise")
        return lin


    def denoise_view(self, r: rd.Renderer, view: int, exposure: float = 1.0, want_linear: bool = False):
        """Filters one batched view of the renderer (accumulation + view G-buffer) into its image."""
        w, h = r._views[view]
        lin = np.zeros((h, w, 4), np.float32) if want_linear else None
        self._check(self.L.wgpt_kpcn_denoise_view(self.h, r.ctx, view, exposure, ptr(lin) if want_linear else None),
                    "denoise_view")
        return lin


WEIGHTS_DIR = Path(__file__).resolve().parent / "weights"


def save_weights(k: Kpcn, path, meta: dict) -> None:
    """Writes the network's FP32 parameters and a JSON description of how they were trained
    (an .npz with arrays `params` and `meta`)."""
    np.savez_compressed(path, params=k.get_params(), meta=np.array(json.dumps(meta)))


def load_weights(k: Kpcn, path) -> dict:
    """Loads parameters written by save_weights into `k`; returns their training description."""
    with np.load(path, allow_pickle=False) as f:
        k.set_params(f["params"])
        return json.loads(str(f["meta"]))


def render_example(scene: sc.Scene, size: int, spp: int, target_spp: int, seed: int = 1, target_seed: int = 977):
    """(noisy accumulation at `spp`, G-buffer, target accumulation at `target_spp`) of one view,
    rendered by the path tracer; the target uses an independent sample stream."""
    scene.camera.aspect = 1.0
    r = rd.Renderer(size, size, seed_fn=lambda: seed)
    r.set_scene(scene, isgbuf=True)
    r.render_gbuffer()
    gbuf = r.read_gbuffer()
    r.reset()
    r.render(tsize=size, reps=spp)
    noisy = r.read_accum()
    r.close()
    t = rd.Renderer(size, size, seed_fn=lambda: target_seed)
    t.set_scene(scene)
    t.render(tsize=size, reps=target_spp)
    target = t.read_accum()
    t.close()
    return noisy, gbuf, target


def tonemap(c: np.ndarray, exposure: float = 1.0) -> np.ndarray:
    """The accumulation pass's display transform (shader.wgsl:2487-2490) in float64."""
    x = np.maximum(np.asarray(c, np.float64)[..., :3], 0.0) * exposure
    return np.power(x / (x + 0.3), 0.4545)


def rmse(a: np.ndarray, b: np.ndarray, exposure: float = 1.0) -> float:
    """RMSE between two linear images in display space (tonemapped, [0, 1])."""
    return float(np.sqrt(np.mean((tonemap(a, exposure) - tonemap(b, exposure)) ** 2)))


def _target_image(t: rd.Renderer, f64: bool) -> np.ndarray:
    """The target renderer's image: its FP64 Welford mean (as rgba32f, alpha 1) or its FP32
    running mean."""
    if not f64:
        return t.read_accum()
    mean, _, _ = t.read_accum_f64()
    out = np.ones(mean.shape[:2] + (4,), np.float32)
    out[..., :3] = mean
    return out


def build_training_set(k: Kpcn, seeds, size: int = 256, spps=(1, 2, 4, 8), target_spp: int = 1024,
                       bounces: int = 4, device: int = 0, pool_paths: int = 1 << 24, target_f64: bool = False) -> int:
    """Adds, for every seeded scene of the small-configuration family, one example per input
    sample count: (progressive accumulation at that count, G-buffer, target at target_spp with
    an independent sample stream, accumulated in FP64 with target_f64).  One renderer pair is
    reused for every scene.  Returns the number of examples added."""
    from . import synth
    n = 0
    t = rd.Renderer(size, size, device=device, seed_fn=lambda: 0)
    r = rd.Renderer(size, size, device=device, seed_fn=lambda: 0)
    t.set_wavefront_config(pool_paths, 0)
    r.set_wavefront_config(pool_paths, 0)
    try:
        for seed in seeds:
            seed = int(seed)
            s = synth.small_scene(seed, size, size, bounces)
            s.camera.aspect = 1.0
            packed = sc.pack_scene_data(s)
            t.seed_fn = lambda: 100_000 + seed
            t.set_scene(s, packed=packed)
            if target_f64:
                t.set_accum_f64(True)
            t.render(tsize=size, reps=target_spp)
            target = _target_image(t, target_f64)
            r.seed_fn = lambda: seed
            r.set_scene(s, isgbuf=True, packed=packed)
            r.render_gbuffer()
            gbuf = r.read_gbuffer()
            r.reset()
            done = 0
            for spp in spps:
                r.render(tsize=size, reps=spp - done)
                done = spp
                k.add_example(r.read_accum(), gbuf, target)
                n += 1
    finally:
        t.close()
        r.close()
    return n


def flagship_family_scene(seed: int, width: int = 1920, height: int = 1080, bounces: int = 8):
    """A scene of the flagship family (seeded instances of the displaced icosphere, analytic
    primitives and Disney materials under the importance-sampled sun sky) seen from a seeded
    camera on a ring around it."""
    import math
    from . import synth
    s = synth.flagship_scene(seed, width, height, bounces)
    rnd = synth.mulberry32(seed * 92821 + 7)
    ang = rnd() * 2.0 * math.pi
    radius = 14.0 + 12.0 * rnd()
    s.camera.position = sc.gm.vec3(radius * math.cos(ang), 2.0 + 8.0 * rnd(), radius * math.sin(ang))
    s.camera.target = sc.gm.vec3(-3.0 + 6.0 * rnd(), 0.5 + 2.5 * rnd(), -3.0 + 6.0 * rnd())
    return s


def crop_origins(seed: int, n: int, width: int, height: int, size: int):
    rnd = np.random.default_rng(seed)
    return [(int(rnd.integers(0, width - size + 1)), int(rnd.integers(0, height - size + 1))) for _ in range(n)]


def build_flagship_training_set(k: Kpcn, seeds, crops: int = 2, size: int = 256, spps=(1, 2, 4, 8),
                                target_spp: int = 1024, bounces: int = 8, width: int = 1920, height: int = 1080,
                                device: int = 0, pool_paths: int = 1 << 24, target_f64: bool = False) -> int:
    """Training examples from the flagship family at the flagship's scale: for each seeded
    scene, `crops` size x size windows of its width x height view are path traced (sections of
    the full image, so objects keep their on-screen size) at every input sample count in
    `spps` (progressively, seed = the scene seed) and at target_spp with an independent stream
    (accumulated in FP64 with target_f64).  One renderer pair is reused for every scene.  Returns
    the number of examples added."""
    tgt_r = rd.Renderer(width, height, device=device, seed_fn=lambda: 0)
    in_r = rd.Renderer(width, height, device=device, seed_fn=lambda: 0)
    tgt_r.set_wavefront_config(pool_paths, 0)
    in_r.set_wavefront_config(pool_paths, 0)
    n = 0
    try:
        for seed in seeds:
            seed = int(seed)
            s = flagship_family_scene(seed, width, height, bounces)
            packed = sc.pack_scene_data(s)
            wins = crop_origins(seed, crops, width, height, size)
            tgt_r.seed_fn = lambda: 100_000 + seed
            tgt_r.set_scene(s, packed=packed)
            if target_f64:
                tgt_r.set_accum_f64(True)
            for (cx, cy) in wins:
                tgt_r.render_section(0, target_spp, cx, cy, size, size)
            tgt_r.synchronize()
            target = _target_image(tgt_r, target_f64)
            in_r.seed_fn = lambda: seed
            in_r.set_scene(s, isgbuf=True, packed=packed)
            in_r.render_gbuffer()
            gbuf = in_r.read_gbuffer()
            done = 0
            for spp in spps:
                for (cx, cy) in wins:
                    in_r.render_section(done, spp - done, cx, cy, size, size)
                in_r.synchronize()
                done = spp
                acc = in_r.read_accum()
                for (cx, cy) in wins:
                    win = (slice(cy, cy + size), slice(cx, cx + size))
                    k.add_example(acc[win], gbuf[win], target[win])
                    n += 1
    finally:
        tgt_r.close()
        in_r.close()
    return n


def gemm_flops(width: int, height: int) -> int:
    """Tensor-core FLOPs of one inference at width x height (padded channel counts, as executed)."""
    h, w = [height], [width]
    for _ in range(4):
        h.append((h[-1] + 1) // 2)
        w.append((w[-1] + 1) // 2)
    return sum(2 * h[l.level] * w[l.level] * l.cout * l.taps * l.cin for l in LAYERS)


def train_data_parallel(k, steps: int, batch: int = 8, crop: int = 64, lr: float = 1e-3, seed: int = 1,
                        device=None) -> np.ndarray:
    """Data-parallel training over the ranks of the default torch.distributed group (one
    process per GPU, NCCL): every rank draws its own crops from its own examples, the
    gradients are summed by all_reduce and every rank applies the same Adam step with the
    mean, so the weights stay identical.  Rank 0's weights are broadcast first.  `k` provides
    n_params, get_params/set_params, grads(batch, crop, seed, buf) and apply(buf, scale, lr)
    (a Kpcn).  Returns the losses averaged over ranks, one per step."""
    import torch
    import torch.distributed as dist
    on = dist.is_available() and dist.is_initialized()
    world = dist.get_world_size() if on else 1
    rank = dist.get_rank() if on else 0
    device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    if world > 1:
        w = torch.from_numpy(k.get_params()).to(device)
        dist.broadcast(w, 0)
        k.set_params(w.cpu().numpy())
    g = torch.empty(k.n_params, dtype=torch.float32, device=device)
    losses = np.zeros(steps, np.float32)
    lv = torch.zeros(1, dtype=torch.float32, device=device)
    for step in range(steps):
        lv[0] = k.grads(batch, crop, (seed * 1_000_003 + step) * world + rank, g)
        if world > 1:
            dist.all_reduce(g)
            dist.all_reduce(lv)
            if device.type == "cuda":
                torch.cuda.current_stream(device).synchronize()
        k.apply(g, 1.0 / world, lr)
        losses[step] = float(lv[0]) / world
    return losses
