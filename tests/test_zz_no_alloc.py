"""The allocation-free denoiser (wgpt_denoise_noalloc) against the context denoiser.

Some callers cannot allocate GPU memory at the point they denoise: a stream being captured into
a CUDA graph (allocation is refused during capture), a host with a fixed memory budget, a
real-time loop that must not wait on the allocator.  wgpt_denoise_noalloc serves them from a
static device array.  This test renders a small scene, denoises it with wgpt_denoise (which uses
context-owned buffers), then calls the allocation-free entry point twice in a row on device
copies of the same inputs and requires the same results (bit for bit, and within the 1e-5
relative bar of the denoiser tests).  This file is collected last on purpose.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from webgpuraytracer_b200 import renderer as rd
from webgpuraytracer_b200 import synth
from webgpuraytracer_b200._lib import NOALLOC_MAX_PIXELS, lib, ptr

pytestmark = pytest.mark.gpu


def test_noalloc_denoise_matches_context_denoise_twice():
    import torch

    w, h = 320, 180
    assert w * h <= NOALLOC_MAX_PIXELS
    scene = synth.small_scene(1, w, h, 4)
    scene.camera.aspect = w / h
    r = rd.Renderer(w, h)
    r.set_scene(scene, isgbuf=True)
    r.render_gbuffer()
    r.render(tsize=320, reps=4)
    color = r.read_accum()
    gbuf = r.read_gbuffer()
    u = rd.denoise_uniforms(w, h, passes=5)
    steps = rd.step_schedule(5, "intended")
    r._check(r.L.wgpt_denoise(r.ctx, ptr(u), ptr(steps), 5), "denoise")
    r.synchronize()
    ref_f = np.empty((h, w, 4), np.float32)
    ref_c = np.empty((h, w, 4), np.float32)
    r._check(r.L.wgpt_read_denoised(r.ctx, ptr(ref_f), ptr(ref_c)), "read_denoised")
    ref_out = r.read_output()
    r.close()

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    d_color = torch.from_numpy(color).to(dev)
    d_gbuf = torch.from_numpy(gbuf).to(dev)
    d_out = torch.empty((h, w, 4), dtype=torch.uint8, device=dev)
    d_comp = torch.empty((h, w, 4), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    L = lib()
    for call in range(2):
        d_out.fill_(7)                      # stale values would show up as mismatches
        d_comp.fill_(float("nan"))
        rc = L.wgpt_denoise_noalloc(d_color.data_ptr(), d_gbuf.data_ptr(), ptr(u), ptr(steps), 5,
                                    d_out.data_ptr(), d_comp.data_ptr(), C.c_void_p(stream.cuda_stream))
        assert rc == 0, f"call {call}: status {rc}"
        torch.cuda.synchronize(dev)
        out = d_out.cpu().numpy()
        comp = d_comp.cpu().numpy()
        np.testing.assert_allclose(comp, ref_c, rtol=1e-5, atol=1e-7)
        np.testing.assert_array_equal(comp, ref_c)
        np.testing.assert_array_equal(out, ref_out)


def test_noalloc_denoise_rejects_images_above_its_limit():
    import torch

    dev = torch.device("cuda", 0)
    small = torch.zeros(16, dtype=torch.float32, device=dev)
    u = rd.denoise_uniforms(512, 512, passes=2)          # 262,144 pixels > the static capacity
    steps = rd.step_schedule(2, "intended")
    rc = lib().wgpt_denoise_noalloc(small.data_ptr(), small.data_ptr(), ptr(u), ptr(steps), 2,
                                    small.data_ptr(), None, None)
    assert rc == 9        # WGPT_E_TOO_LARGE, nothing queued
    assert torch.count_nonzero(small).item() == 0


def test_noalloc_denoise_rejects_misaligned_pointers():
    import torch

    dev = torch.device("cuda", 0)
    buf = torch.zeros(4096, dtype=torch.float32, device=dev)
    base = buf.data_ptr()
    u = rd.denoise_uniforms(16, 16, passes=1)
    steps = rd.step_schedule(1, "intended")
    L = lib()
    # colour, G-buffer and the float output are read and written as float4, the rgba8 output as uchar4
    for color, gbuf, out8, comp in ((base + 4, base, base, None), (base, base + 8, base, None),
                                    (base, base, base, base + 4), (base, base, base + 2, None)):
        rc = L.wgpt_denoise_noalloc(color, gbuf, ptr(u), ptr(steps), 1, out8, comp, None)
        assert rc == 1      # WGPT_E_INVALID, nothing queued
    torch.cuda.synchronize(dev)
    assert torch.count_nonzero(buf).item() == 0
