"""Failure containment and recovery on the GPU, without faulting it.

* The tensor-core kernels' bounded mbarrier wait gives up on a phase that nothing completes and
  reports the timeout bit; the device stays usable (a GEMM runs afterwards).
* The host watchdog returns control while a long render is still queued.
* NaN transformation matrices in the scene (host-side injection) render without a device error
  and exactly as the oracle renders them.
* Checkpoint / resume: an accumulation saved after some samples and restored into a fresh
  renderer continues bit for bit like an uninterrupted render, FP64 records included.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import oracle
from webgpuraytracer_b200 import _lib
from webgpuraytracer_b200 import renderer as rd
from webgpuraytracer_b200 import scene as sc
from webgpuraytracer_b200 import synth

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_and_device_stays_usable():
    L = _lib.lib()
    status = np.zeros(1, np.uint32)
    ms = np.zeros(1, np.float32)
    assert L.wgpt_selftest_wait(0, 1 << 14, _lib.ptr(status), _lib.ptr(ms)) == 0
    assert status[0] == 4                      # ERR_TC_TIMEOUT from the device
    assert 0.0 < ms[0] < 5000.0
    a = np.full((128, 32), 0x3F80, np.uint16)  # bf16 1.0
    b = np.full((32, 32), 0x3F80, np.uint16)
    c = np.zeros((128, 32), np.float32)
    assert L.wgpt_gemm_bf16(0, _lib.ptr(a), _lib.ptr(b), _lib.ptr(c), 128, 32, 32) == 0
    assert np.all(c == 32.0)


def test_watchdog_returns_while_work_runs():
    s = synth.flagship_scene(1, 1920, 1080, 8, instances=8, prims=8, subdivisions=4)
    r = rd.Renderer(1920, 1080)
    r.set_scene(s)
    r.render(tsize=1920, reps=32, sync=False)
    assert r.wait(0) is False                  # still queued: the host gets control back
    assert r.wait(120_000) is True
    assert np.isfinite(r.read_accum()).all()
    r.close()


def test_nan_matrices_are_contained():
    s = synth.small_scene(2, 96, 96, 4)
    p = sc.pack_scene_data(s)
    objs = np.ascontiguousarray(p.objects).view(np.float32).reshape(-1, 24).copy()
    objs[1, :16] = np.nan                      # one object's inverse matrix
    bad = sc.PackedScene(**{**p.__dict__})
    bad.objects = objs.view(np.uint8).reshape(-1)
    s.camera.aspect = 1.0
    s.camera.update_rays2()
    params = sc.pack_params(s, bad, 96, 96, 0, 1, (0, 0))
    acc_o = np.zeros((96, 96, 4), np.float32)
    out_o = np.zeros((96, 96, 4), np.uint8)
    assert oracle.render(oracle.OracleScene(bad), params, 0, 4, (0, 0, 96, 96), acc_o, out_o,
                         oracle.default_threads()) == 0
    r = rd.Renderer(96, 96)
    r.set_scene(s, packed=bad)
    r._check(r.L.wgpt_set_params(r.ctx, rd.ptr(params)), "set_params")
    r._check(r.L.wgpt_render(r.ctx, 0, 4, 0, 0, 96, 96), "render")
    r.synchronize()                            # no device error
    acc_g = r.read_accum()
    same = (acc_g == acc_o) | (np.isnan(acc_g) & np.isnan(acc_o))
    assert same.all()
    r.close()


def test_checkpoint_resume_is_bitexact(tmp_path):
    s = synth.small_scene(3, 128, 96, 4)
    s.camera.aspect = 128 / 96

    def fresh():
        r = rd.Renderer(128, 96)
        r.set_scene(s)
        r.set_accum_f64(True)
        return r

    whole = fresh()
    whole.render(tsize=128, reps=8)
    first = fresh()
    first.render(tsize=128, reps=4)
    path = tmp_path / "ckpt.npz"
    first.save_state(path)
    first.close()
    resumed = fresh()
    resumed.load_state(path)
    assert resumed.frame == 4
    resumed.render(tsize=128, reps=4)
    assert np.array_equal(resumed.read_accum(), whole.read_accum())
    a = np.empty((96, 128, 8), np.float64)
    b = np.empty((96, 128, 8), np.float64)
    resumed._check(resumed.L.wgpt_read_accum_f64(resumed.ctx, rd.ptr(a)), "f64")
    whole._check(whole.L.wgpt_read_accum_f64(whole.ctx, rd.ptr(b)), "f64")
    assert np.array_equal(a, b)
    other = rd.Renderer(64, 64)
    other.set_scene(s)
    with pytest.raises(ValueError):
        other.load_state(path)
    for r in (whole, resumed, other):
        r.close()


def test_l2_probe_measures_more_than_hbm_can_stream():
    L = _lib.lib()
    out = C.c_double(0.0)
    assert L.wgpt_probe_l2_read(0, 32 << 20, 50, C.byref(out)) == 0
    assert 1000.0 < out.value < 200000.0                 # GB/s: an L2-resident read, finite
