"""Benchmark of the progressive path tracer on the flagship workload.

Workload: the two-level-BVH, full-Disney-BSDF scene at 1920x1080 with 8 bounces (a displaced
81,920-triangle icosphere instanced 64x, 32 analytic primitives, a 2048x1024 RGBE sky with
importance sampling), seed 1.  One step = one render call of 64 progressive samples per pixel
(64 x 2,073,600 = 132,710,400 camera paths) through the renderer's C ABI, like
Renderer.render with reps = 64 in tracer.js (sample_number = frame .. frame + 63).  The metric
is paths/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N>1 runs under torchrun, one process per GPU; every rank renders the same view with its own
seed (independent sample streams of one progressive image, no data-path collective), and the
job's value is all ranks' paths over the slowest rank's device time.  `--impl reference` times
the CPU restatement of the reference's shaders on this host's cores on the same workload (the
reference's WGSL cannot run here: it needs a WebGPU device and no graphics stack exists).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WIDTH, HEIGHT, BOUNCES, SPP = 1920, 1080, 8, 64
METRIC = "paths/s (1920x1080, 8 bounces)"
PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}   # earlier measurement on this pool

# Algorithmic bytes per counted unit (counter slots of wgpt_read_counters): what the reference's
# algorithm must read or write per unit of work, independent of how it is laid out.
BYTES_PER_UNIT = {
    3: 32,    # BVH node popped (two 16-byte vectors)
    4: 32,    # child AABB tested
    5: 48,    # triangle tested (v0, v1, v2)
    6: 96,    # TLAS object visited (matrix + header)
    7: 144,   # shading event (material record)
    9: 4,     # environment CDF probe
    10: 8,    # sky texel read (rgba16f)
    11: 32,   # hit attributes of the winning primitive (normals)
}
PIXEL_BYTES = 16 + 16 + 4   # accumulation read + write, rgba8 store
# DRAM bytes (read + write) per closest-hit ray of this workload, from ncu captures of this
# workload (bench.py cannot run ncu itself): 2,077 MB per steady-state launch of an
# 8,388,608-slot pool (every slot holds a live path while units remain, so 8,388,608 rays per
# launch; mean of launches 13-15: 248 B per ray); a 2,097,152-slot pool gives 250 B per ray, so
# the traffic scales with the rays, not the pool.  A launch's traffic is this times its rays.
EXTEND_DRAM_BYTES_PER_RAY = 2.0771e9 / 8_388_608
KERNELS = ["k_wf_fill", "k_wf_extend", "k_wf_shade", "k_wf_shadow", "k_wf_resolve", "k_wf_shade_miss",
           "k_wf_accumulate", "k_wf_control"]


def algorithmic_bytes(counters: np.ndarray, pixels: int) -> float:
    return float(sum(int(counters[k]) * b for k, b in BYTES_PER_UNIT.items()) + pixels * PIXEL_BYTES)


def stage_bytes(stage_counters: np.ndarray, pixels: int, megakernel: bool) -> list[float]:
    """Algorithmic bytes per stage; the accumulation traffic belongs to the stage that writes it."""
    out = []
    for st in range(8):
        c = stage_counters[st]
        px = pixels if (st == 6 or (st == 0 and megakernel)) else 0
        out.append(algorithmic_bytes(c, px))
    return out


def load_peaks() -> tuple[dict, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text()), "measured"
    return PEAKS_FALLBACK, "fallback"


class ClockSampler:
    """nvidia-smi clock and throttle-reason samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in Path(self.path).read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup(n_gpus: int):
    from webgpuraytracer_b200 import replicas
    return replicas.setup("nccl")


def max_over_ranks(x: float, world: int) -> float:
    from webgpuraytracer_b200 import replicas
    return replicas.max_over_ranks(x, world)


def barrier(world: int):
    from webgpuraytracer_b200 import replicas
    replicas.barrier(world)


def replicas_seed(rank: int) -> int:
    from webgpuraytracer_b200 import replicas
    return replicas.rank_seed(1, rank)


def build_workload(seed: int = 1):
    from webgpuraytracer_b200 import scene as sc
    from webgpuraytracer_b200 import synth
    s = synth.flagship_scene(seed, WIDTH, HEIGHT, BOUNCES)
    return s, sc.pack_scene_data(s)


def cpu_sample(scene, packed, frames: int, min_seconds: float, max_frames: int, rows: int | None = None):
    """Times the CPU restatement on all host cores: whole 1080p frames (or the first `rows` rows)
    one sample per pixel, until min_seconds have passed or max_frames were rendered."""
    import oracle
    from webgpuraytracer_b200 import scene as sc
    scene.camera.update_rays2()
    params = sc.pack_params(scene, packed, WIDTH, HEIGHT, 0, 1)
    os_ = oracle.OracleScene(packed)
    h = rows or HEIGHT
    acc = np.zeros((HEIGHT, WIDTH, 4), np.float32)
    out = np.zeros((HEIGHT, WIDTH, 4), np.uint8)
    threads = os.cpu_count() or 1
    done = 0
    t0 = time.perf_counter()
    while done < max_frames and (done < frames or time.perf_counter() - t0 < min_seconds):
        oracle.render(os_, params, done, 1, (0, 0, WIDTH, h), acc, out, threads)
        done += 1
    dt = time.perf_counter() - t0
    return WIDTH * h * done / dt, threads, f"{done} x {WIDTH}x{h} frame(s) at 1 spp, {dt:.1f} s"


def run_reference(args):
    """--impl reference: the CPU restatement of the reference's shaders on every host core."""
    rank, world, _ = int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), 0
    if rank != 0:
        return 0
    scene, packed = build_workload()
    import oracle
    from webgpuraytracer_b200 import scene as sc
    scene.camera.update_rays2()
    params = sc.pack_params(scene, packed, WIDTH, HEIGHT, 0, 1)
    os_ = oracle.OracleScene(packed)
    acc = np.zeros((HEIGHT, WIDTH, 4), np.float32)
    out = np.zeros((HEIGHT, WIDTH, 4), np.uint8)
    threads = os.cpu_count() or 1
    # one step = the whole 1080p frame at 1 spp (2,073,600 paths; a fraction of a second on the
    # host's cores), sample numbers advancing like the reference's frames
    def step(i):
        oracle.render(os_, params, i, 1, (0, 0, WIDTH, HEIGHT), acc, out, threads)

    for i in range(args.warmup):
        step(i)
    t0 = time.perf_counter()
    for i in range(args.steps):
        step(args.warmup + i)
    dt = time.perf_counter() - t0
    paths = WIDTH * HEIGHT * args.steps
    value = paths / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "paths/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded scene generator)",
        "config": {"workload": "flagship 1920x1080, 8 bounces, 64 instances x 81,920-tri BLAS + 32 prims, 2048x1024 RGBE env",
                   "step": f"one {WIDTH}x{HEIGHT} frame at 1 spp", "l2": "not applicable (CPU)"},
        "cpu_baseline": {"value": value, "unit": "paths/s", "cores": threads, "kind": "port",
                         "sample": f"{args.steps} {WIDTH}x{HEIGHT} frames at 1 spp"},
        "e2e": {"value": value, "unit": "paths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference's WGSL needs a WebGPU device; no graphics stack exists on this box, so the "
                "reference arm is the CPU restatement of shader.wgsl (OpenMP over pixels)",
    }
    print(json.dumps(line), flush=True)
    return 0


def stage_report(r, rd, launch_once, stream, flush, paths_per_step: int, mega: bool) -> dict:
    """Per-stage launch times of one step (event pair around every stage launch; the iteration
    loop is then driven from the host instead of the graph: same kernels, same stream) and the
    work counters of one step (a separate counting pass), both outside the timed region."""
    import torch
    r._check(r.L.wgpt_set_stage_timing(r.ctx, 1), "stage timing")
    with torch.cuda.stream(stream):
        flush.fill_(0.5)
    launch_once()
    r.synchronize()
    stage_ms = np.zeros(8, np.float64)
    stage_launches = np.zeros(8, np.uint32)
    r._check(r.L.wgpt_read_stage_times(r.ctx, rd.ptr(stage_ms), rd.ptr(stage_launches)), "stage times")
    r._check(r.L.wgpt_set_stage_timing(r.ctx, 0), "stage timing")
    r.set_counting(True)
    launch_once()
    cnt = r.read_counters()
    stage_cnt = np.zeros(128, np.uint64)
    r._check(r.L.wgpt_read_stage_counters(r.ctx, rd.ptr(stage_cnt)), "stage counters")
    r.set_counting(False)
    sbytes = stage_bytes(stage_cnt.reshape(8, 16), paths_per_step, mega)
    dom = int(np.argmax(stage_ms))
    bytes_per_launch = sbytes[dom] / max(1, int(stage_launches[dom]))
    avg_launch_s = stage_ms[dom] / 1e3 / max(1, int(stage_launches[dom]))
    stages = {}
    for st in range(8):
        if stage_launches[st]:
            t = stage_ms[st] / 1e3
            stages[("k_render" if mega else KERNELS[st])] = {
                "launches": int(stage_launches[st]), "ms_total": float(stage_ms[st]),
                "share": float(stage_ms[st] / stage_ms.sum()), "algorithmic_GBps": sbytes[st] / t / 1e9 if t else None}
    # the graph runs the same kernels the timing pass launched from the host (fill, 6 per
    # iteration, accumulate)
    return {"stages": stages, "achieved": bytes_per_launch / avg_launch_s / 1e9, "bytes_per_launch": bytes_per_launch,
            "avg_launch_s": avg_launch_s, "dom": dom, "cnt": cnt, "launches": int(stage_launches.sum())}


# The plain method's filter candidates: the reference Denoiser's defaults (tracer.js:2424-2435)
# with its own 4 passes as it runs (every pass at step 8) and as its loop intends (1, 2, 4, 8), and
# the a-trous configuration's 5 passes (1..16).  The plain arm takes the best of them and of no
# filter at every sample count.
ATROUS_ARMS = {"atrous_4_as_run": (4, "as_run"), "atrous_4": (4, "intended"), "atrous_5": (5, "intended")}


def time_to_rmse(args) -> dict:
    """Time to display-space RMSE <= threshold against an FP64-accumulated reference of
    --ref-spp samples, on the flagship workload itself (1920x1080, 8 bounces, seed 1, the bench's
    scene and camera): plain accumulation plus the a-trous filter against accumulation plus the
    learned denoiser.  The network's weights were trained on the GPU by train_denoiser from pairs
    this tracer renders (the package's flagship weights, whose recipe is stored with them), or
    with --kpcn-train here: flagship-family scenes (seeds 1000.., their own cameras) as 256x256
    windows of their 1080p views, inputs at --kpcn-spps, targets at --kpcn-target-spp with an
    independent stream.  The flagship scene and the held-out evaluation scenes (seeds 5000..) are
    not trained on."""
    import torch
    from webgpuraytracer_b200 import kpcn, train_denoiser
    from webgpuraytracer_b200 import renderer as rd
    from webgpuraytracer_b200 import scene as sc
    W, H, thr = WIDTH, HEIGHT, args.rmse_threshold
    out = {"threshold": thr, "space": "display (shader.wgsl tonemap, exposure 1); linear RMSE reported beside it",
           "scene": f"flagship workload, seed 1, {W}x{H}, {BOUNCES} bounces (held out of training)",
           "reference": f"{args.ref_spp} spp, FP64 Welford accumulation"}
    k = kpcn.Kpcn(0, seed=1)
    weights = Path(args.kpcn_weights) if args.kpcn_weights else kpcn.WEIGHTS_DIR / "kpcn_flagship.npz"
    if weights.exists() and not args.kpcn_train:
        # weights trained on the GPU by train_denoiser (the recipe travels inside the file)
        meta = kpcn.load_weights(k, weights)
        out["training"] = {"source": "pretrained", "file": str(weights.relative_to(ROOT))
                           if weights.is_relative_to(ROOT) else str(weights), "params": k.n_params, **meta}
    else:
        t0 = time.perf_counter()
        spps = tuple(int(v) for v in args.kpcn_spps.split(","))
        n_ex = kpcn.build_flagship_training_set(k, range(1000, 1000 + args.kpcn_scenes), crops=args.kpcn_crops,
                                                spps=spps, target_spp=args.kpcn_target_spp, bounces=BOUNCES)
        t_data = time.perf_counter() - t0
        t0 = time.perf_counter()
        losses = train_denoiser.train(k, args.kpcn_steps, 16, 128, 1e-3, args.kpcn_schedule)
        t_train = time.perf_counter() - t0
        out["training"] = {"source": "trained in this run",
                           "family": "flagship (seeded instances, primitives, Disney materials, sun sky, seeded cameras)",
                           "scenes": args.kpcn_scenes, "windows_per_scene": args.kpcn_crops,
                           "window": "256x256 of 1920x1080", "examples": n_ex, "input_spp": list(spps),
                           "target_spp": args.kpcn_target_spp, "steps": args.kpcn_steps, "schedule": args.kpcn_schedule,
                           "batch": "16 x 128^2 crops", "data_s": t_data, "train_s": t_train,
                           "loss_first_50": float(np.mean(losses[:50])), "loss_last_50": float(np.mean(losses[-50:])),
                           "params": k.n_params}
    out["held_out"] = held_out_eval(k, args)

    scene, packed = build_workload()
    ref_r = rd.Renderer(W, H, seed_fn=lambda: 4242)
    ref_r.set_scene(scene, packed=packed)
    ref_r.set_accum_f64(True)
    done = 0
    t0 = time.perf_counter()
    while done < args.ref_spp:
        n = min(4096, args.ref_spp - done)
        ref_r.render(tsize=W, reps=n)
        done += n
    ref, var, _ = ref_r.read_accum_f64()
    out["reference_s"] = time.perf_counter() - t0
    ref_r.close()
    ref_disp = kpcn.tonemap(ref)
    # the reference's own noise in display space (delta method: derivative of the tonemap times
    # the standard error of each pixel mean)
    x = np.maximum(ref, 0.0)
    deriv = 0.4545 * (x / (x + 0.3)) ** (0.4545 - 1.0) * 0.3 / (x + 0.3) ** 2
    out["reference_display_noise_rmse"] = float(np.sqrt(np.mean(deriv ** 2 * var / args.ref_spp)))

    def disp_rmse(d):
        return float(np.sqrt(np.mean((np.clip(d[..., :3], 0.0, 1.0) - ref_disp) ** 2)))

    def lin_rmse(lin):
        return float(np.sqrt(np.mean((np.asarray(lin, np.float64)[..., :3] - ref) ** 2)))

    ev = rd.Renderer(W, H, seed_fn=lambda: 7)
    ev.set_scene(scene, isgbuf=True, packed=packed)
    ev.render_gbuffer()
    ev.reset()
    dens = {name: rd.Denoiser(ev, passes=pp, mode=mode) for name, (pp, mode) in ATROUS_ARMS.items()}
    sweep, done, spp = [], 0, 1
    while spp <= args.max_spp:
        ev.render(tsize=W, reps=spp - done)
        done = spp
        acc = ev.read_accum()
        row = {"spp": spp, "accum": kpcn.rmse(acc, ref), "accum_linear": lin_rmse(acc)}
        for name, dn in dens.items():
            dn.execute()
            row[name] = disp_rmse(dn.read()[1])
        if spp <= args.max_nn_spp:
            lin = k.denoise(ev)
            row["kpcn"] = kpcn.rmse(lin, ref)
            row["kpcn_linear"] = lin_rmse(lin)
        sweep.append(row)
        plain_best = min(row[c] for c in ("accum", *ATROUS_ARMS))
        if plain_best <= thr:
            break
        spp *= 2
    ev.close()
    out["sweep"] = sweep

    def first(key_fn):
        for row in sweep:
            v = key_fn(row)
            if v is not None and v <= thr:
                return row
        return None

    row_p = first(lambda r_: min(r_[c] for c in ("accum", *ATROUS_ARMS)))
    row_n = first(lambda r_: r_.get("kpcn"))

    def timed(spp_, filt):
        """Device time of rendering spp_ samples from frame 0 and filtering once, on a renderer
        that has already run one call of the same size (its path pool and sample buffer are
        allocated and its loop graph built, as in an interactive session); frame 0 overwrites
        the accumulation, so the timed images equal a fresh renderer's."""
        r_ = rd.Renderer(W, H, seed_fn=lambda: 7)
        r_.set_scene(scene, isgbuf=True, packed=packed)
        r_.render_gbuffer()
        r_.reset()
        r_.render(tsize=W, reps=spp_)
        r_.reset()
        st = torch.cuda.ExternalStream(r_.stream_handle())
        dn = rd.Denoiser(r_, passes=ATROUS_ARMS[filt][0], mode=ATROUS_ARMS[filt][1]) if filt in ATROUS_ARMS else None
        if dn:
            dn.execute()                      # allocates the filter's buffers outside the timing
        if filt == "kpcn":
            k.denoise(r_, want_linear=False)
        r_.synchronize()
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record(st)
        r_.render(tsize=W, reps=spp_, sync=False)
        e1.record(st)
        if dn:
            dn.execute()
        elif filt == "kpcn":
            k.denoise(r_, want_linear=False)
        e2.record(st)
        r_.synchronize()
        torch.cuda.synchronize()
        r_.close()
        return e0.elapsed_time(e1), e1.elapsed_time(e2)

    def arm(row, candidates, label):
        if row is None:
            last = [r_ for r_ in sweep if any(c in r_ for c in candidates)][-1]
            best = min((c for c in candidates if c in last), key=lambda c: last[c])
            s_est = last["spp"] * (last[best] / thr) ** 2
            r_ms, f_ms = timed(last["spp"], best)
            return {"spp": None, "spp_extrapolated": s_est, "ms": r_ms * s_est / last["spp"] + f_ms,
                    "method": f"{best} (1/sqrt(spp) extrapolation of the last sweep point)", "arm": label}
        best = min((c for c in candidates if c in row and row[c] <= thr), key=lambda c: row[c])
        r_ms, f_ms = timed(row["spp"], best)
        return {"spp": row["spp"], "ms": r_ms + f_ms, "render_ms": r_ms, "filter_ms": f_ms, "method": best,
                "rmse": row[best], "arm": label}

    out["plain"] = arm(row_p, ("accum", *ATROUS_ARMS), "accumulation + a-trous (best filter per sample count)")
    out["neural"] = arm(row_n, ("kpcn",), "accumulation + learned denoiser")
    if out["plain"]["ms"] and out["neural"]["ms"]:
        out["plain_over_neural"] = out["plain"]["ms"] / out["neural"]["ms"]
    # inference throughput at 1080p on the tensor cores
    r_ = rd.Renderer(W, H, seed_fn=lambda: 7)
    r_.set_scene(scene, isgbuf=True, packed=packed)
    r_.render_gbuffer()
    r_.reset()
    r_.render(tsize=W, reps=1)
    st = torch.cuda.ExternalStream(r_.stream_handle())
    for _ in range(3):
        k.denoise(r_, want_linear=False)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    reps = 10
    for _ in range(reps):
        k.denoise(r_, want_linear=False)
    e1.record(st)
    r_.synchronize()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    flops = kpcn.gemm_flops(W, H)
    peaks, kind = load_peaks()
    tf = flops / (ms / 1e3) / 1e12
    out["kpcn_inference_1080p"] = {"ms": ms, "gemm_tflops": tf, "gemm_flops": flops,
                                   "frac_of_bf16_peak": tf / peaks["bf16_tflops"] if "bf16_tflops" in peaks else None,
                                   "peak_source": "measured (MEASURED_PEAKS.json bf16_tflops)" if kind == "measured"
                                   else "fallback 1.59 PFLOP/s"}
    r_.close()
    k.close()
    return out


def held_out_eval(k, args, n_scenes: int = 16, size: int = 256, spps=(4, 8, 16), target_spp: int = 4096,
                  margin: int = 32) -> dict:
    """Display RMSE of the noisy input, the a-trous filter (the a-trous configuration's 5
    passes) and the network on one 256x256 window of each of n_scenes flagship-family scenes
    that training never saw (seeds 5000..), at each input sample count, against a target_spp
    render with an independent stream.  The input is rendered as a section of the scene's
    1920x1080 view reaching `margin` pixels beyond the window (so both filters see real
    neighbours at the window's edges); both filters run over the image and are scored on the
    window."""
    from webgpuraytracer_b200 import kpcn
    from webgpuraytracer_b200 import renderer as rd
    from webgpuraytracer_b200 import scene as sc
    res = {s_: {"noisy": [], "atrous_5": [], "kpcn": []} for s_ in spps}
    tgt_r = rd.Renderer(WIDTH, HEIGHT, seed_fn=lambda: 0)
    in_r = rd.Renderer(WIDTH, HEIGHT, seed_fn=lambda: 0)
    for r_ in (tgt_r, in_r):
        r_.set_wavefront_config(1 << 24, 0)
    try:
        for seed in range(5000, 5000 + n_scenes):
            s = kpcn.flagship_family_scene(seed, WIDTH, HEIGHT, BOUNCES)
            packed = sc.pack_scene_data(s)
            (cx, cy), = kpcn.crop_origins(seed, 1, WIDTH, HEIGHT, size)
            win = (slice(cy, cy + size), slice(cx, cx + size))
            x0, y0 = max(cx - margin, 0), max(cy - margin, 0)
            x1, y1 = min(cx + size + margin, WIDTH), min(cy + size + margin, HEIGHT)
            tgt_r.seed_fn = lambda: 200_000 + seed
            tgt_r.set_scene(s, packed=packed)
            tgt_r.render_section(0, target_spp, cx, cy, size, size)
            tgt_r.synchronize()
            target = tgt_r.read_accum()[win]
            in_r.seed_fn = lambda: seed
            in_r.set_scene(s, isgbuf=True, packed=packed)
            in_r.render_gbuffer()
            done = 0
            for spp in spps:
                in_r.render_section(done, spp - done, x0, y0, x1 - x0, y1 - y0)
                in_r.synchronize()
                done = spp
                acc = in_r.read_accum()
                res[spp]["noisy"].append(kpcn.rmse(acc[win], target))
                dn = rd.Denoiser(in_r, passes=5)
                dn.execute()
                comp = dn.read()[1][win]
                res[spp]["atrous_5"].append(float(np.sqrt(np.mean(
                    (np.clip(comp[..., :3], 0.0, 1.0) - kpcn.tonemap(target)) ** 2))))
                lin = k.denoise(in_r)
                res[spp]["kpcn"].append(kpcn.rmse(lin[win], target))
    finally:
        tgt_r.close()
        in_r.close()
    return {"scenes": n_scenes, "seeds": f"5000..{5000 + n_scenes - 1}", "window": f"{size}x{size} of 1920x1080",
            "margin": margin, "target_spp": target_spp,
            "mean_display_rmse": {str(s_): {m: float(np.mean(v)) for m, v in d.items()} for s_, d in res.items()},
            "kpcn_better_than_atrous": {str(s_): int(sum(a_ < b_ for a_, b_ in zip(d["kpcn"], d["atrous_5"])))
                                        for s_, d in res.items()}}


# FP32 operations per counted unit for the small configuration's ALU roofline (the constants
# are the operation counts of the restated routines, rounded): slab test of one child box 12,
# Moller-Trumbore 27, one analytic primitive (ray transform + quadric) 40, one shading event
# (lobe probabilities, sampling, eval and pdf of the Disney BSDF, NEE set-up) 300, one CDF probe 2.
FLOPS_PER_UNIT = {4: 12, 5: 27, 6: 40, 7: 300, 9: 2}
FP32_PEAK_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12   # 148 SMs x 128 FP32 lanes x FMA x 1965 MHz


def autotune_shapes() -> dict:
    from webgpuraytracer_b200 import autotune
    return autotune.TRAV_SHAPES


def small_config(steps: int = 20, warmup: int = 3) -> dict:
    """The small configuration (256x256, 16 spp, 4 bounces, 8 analytic primitives, constant sky)
    on the GPU: paths/s over whole 16-spp calls and the FP32 SIMT rate of the counted work
    against the FP32 peak.  Inputs stay resident; each step is one render call."""
    import torch
    from webgpuraytracer_b200 import renderer as rd
    from webgpuraytracer_b200 import scene as sc
    from webgpuraytracer_b200 import synth
    w = h = 256
    spp = 16
    s = synth.small_scene(1, w, h, 4)
    packed = sc.pack_scene_data(s)
    r = rd.Renderer(w, h, seed_fn=lambda: 1)
    r.set_scene(s, packed=packed)
    s.camera.update_rays2()
    st = torch.cuda.ExternalStream(r.stream_handle())

    def launch(i):
        p_ = sc.pack_params(s, packed, w, h, i * spp, 1)
        r._check(r.L.wgpt_set_params(r.ctx, rd.ptr(p_)), "params")
        r._check(r.L.wgpt_render(r.ctx, i * spp, spp, 0, 0, w, h), "render")

    for i in range(warmup):
        launch(i)
    r.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for i in range(steps):
        launch(warmup + i)
    e1.record(st)
    r.synchronize()
    torch.cuda.synchronize()
    sec = e0.elapsed_time(e1) / 1e3
    r.set_counting(True)
    launch(warmup)
    cnt = r.read_counters()
    r.set_counting(False)
    r.close()
    flops = float(sum(int(cnt[k]) * f for k, f in FLOPS_PER_UNIT.items()))
    tf = flops * steps / sec / 1e12
    return {"workload": "small 256x256, 16 spp, 4 bounces, 8 primitives, constant sky (one render call per step)",
            "paths_per_s": w * h * spp * steps / sec, "ms_per_step": sec / steps * 1e3,
            "rays_per_s": float(cnt[1] + cnt[2]) * steps / sec,
            "fp32_roofline": {"bound": "fp32 simt", "achieved": tf, "peak": FP32_PEAK_TFLOPS, "unit": "TFLOP/s",
                              "frac": tf / FP32_PEAK_TFLOPS, "flops_per_step": flops,
                              "peak_source": "nominal: 148 SMs x 128 FP32 lanes x 2 (FMA) x 1965 MHz; the kernels "
                                             "are built without multiply-add contraction, so 0.5 is their ceiling"}}


def cpu_atrous_baseline(passes: int = 5) -> dict:
    """The a-trous configuration (1920x1080, 5 passes, the Denoiser defaults) through the CPU
    restatement of denoiser.wgsl on every host core: ms per frame."""
    import oracle
    from webgpuraytracer_b200 import renderer as rd
    rng = np.random.default_rng(1)
    w, h = WIDTH, HEIGHT
    color = (np.abs(rng.standard_normal((h, w, 4))) * 0.5).astype(np.float32)
    gbuf = rng.standard_normal((h, w, 12)).astype(np.float32)
    gbuf[..., 11] = np.abs(gbuf[..., 11]) * 5.0
    u = rd.denoise_uniforms(w, h, passes=passes)
    steps = rd.step_schedule(passes, "intended")
    threads = os.cpu_count() or 1
    oracle.denoise(color, gbuf, u, steps, threads)
    t0 = time.perf_counter()
    reps = 2
    for _ in range(reps):
        oracle.denoise(color, gbuf, u, steps, threads)
    ms = (time.perf_counter() - t0) / reps * 1e3
    return {"ms_per_frame": ms, "cores": threads, "kind": "port",
            "sample": f"{reps} frames of 1920x1080, {passes} passes (steps 1..16), seeded synthetic buffers"}


def run_ours(args):
    rank, world, local = dist_setup(args.gpus)
    import torch
    from webgpuraytracer_b200 import renderer as rd
    from webgpuraytracer_b200 import scene as sc

    torch.cuda.set_device(local)
    scene, packed = build_workload()
    r = rd.Renderer(WIDTH, HEIGHT, device=local, seed_fn=lambda: replicas_seed(rank))
    r.set_scene(scene, packed=packed)
    mega = args.mode == "megakernel"
    r._check(r.L.wgpt_set_render_mode(r.ctx, 1 if mega else 0), "render mode")
    if args.pool:
        r.set_wavefront_config(args.pool, 0)
    pool_paths = r.wavefront_config()[0]
    stream = torch.cuda.ExternalStream(r.stream_handle(), device=torch.device("cuda", local))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")   # > 126 MB L2
    scene.camera.update_rays2()
    spp = args.spp

    def launch(step):
        frame = step * spp
        p = sc.pack_params(scene, packed, WIDTH, HEIGHT, frame, replicas_seed(rank))
        r._check(r.L.wgpt_set_params(r.ctx, rd.ptr(p)), "set_params")
        r._check(r.L.wgpt_render(r.ctx, frame, spp, 0, 0, WIDTH, HEIGHT), "render")

    # kernel variants and thresholds by the autotuner (coordinate descent, one render call of the
    # workload per candidate after a warm-up call), unless fixed on the command line
    tuned_k = None
    if not mega and not args.no_tune:
        from webgpuraytracer_b200 import autotune
        tuned_k = autotune.tune_kernels(r, lambda: launch(0))
    # warm-up (builds the loop graph on the first call)
    for i in range(args.warmup):
        launch(i)
    r.synchronize()
    # device-resident timing: one event pair per step on the library's stream, L2 flushed
    # between steps
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    sampler = ClockSampler(local)
    barrier(world)
    torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.3)
    for i in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(float(i))
            starts[i].record(stream)
        launch(args.warmup + i)
        with torch.cuda.stream(stream):
            ends[i].record(stream)
    r.synchronize()
    torch.cuda.synchronize()
    barrier(world)
    clocks = sampler.stop()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    dev_s = sum(step_ms) / 1e3
    dev_s_max = max_over_ranks(dev_s, world)
    paths_per_step = WIDTH * HEIGHT * spp
    value = paths_per_step * args.steps * world / dev_s_max

    # end-to-end through the C ABI with host buffers: params in, rgba8 image out, every step
    out_host = torch.empty((HEIGHT, WIDTH, 4), dtype=torch.uint8, pin_memory=True)
    e2e_steps = max(1, min(args.steps, 16))
    barrier(world)
    t0 = time.perf_counter()
    for i in range(e2e_steps):
        launch(args.warmup + args.steps + i)
        r._check(r.L.wgpt_read_output(r.ctx, out_host.data_ptr()), "read_output")
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    e2e_value = paths_per_step * e2e_steps * world / e2e_s

    rep = stage_report(r, rd, lambda: launch(args.warmup), stream, flush, paths_per_step, mega)
    stages, achieved, bytes_per_launch, avg_launch_s, dom, cnt, launches = (
        rep["stages"], rep["achieved"], rep["bytes_per_launch"], rep["avg_launch_s"], rep["dom"], rep["cnt"],
        rep["launches"])
    peaks, peak_kind = load_peaks()
    rays = int(cnt[1] + cnt[2])
    l2 = C.c_double(0.0)
    r._check(r.L.wgpt_probe_l2_read(local, 64 << 20, 200, C.byref(l2)), "L2 probe")
    ext_rays_per_launch = int(cnt[1]) / max(1, stages.get("k_wf_extend", {}).get("launches", 1))

    # the opt-in alias-table environment sampling on the same steps (statistically equal images,
    # not bit-exact, so never the headline value)
    r.set_env_sampling(rd.ENV_ALIAS)
    for i in range(args.warmup):
        launch(i)
    r.synchronize()
    barrier(world)
    for i in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(float(i))
            starts[i].record(stream)
        launch(args.warmup + i)
        with torch.cuda.stream(stream):
            ends[i].record(stream)
    r.synchronize()
    torch.cuda.synchronize()
    alias_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    alias_s = max_over_ranks(sum(alias_ms) / 1e3, world)
    r.set_env_sampling(rd.ENV_CDF)
    env_alias = {"value": paths_per_step * args.steps * world / alias_s, "unit": "paths/s",
                 "note": "opt-in O(1) alias-table sky sampling on the same steps; images agree statistically "
                         "with the CDF search, not bit for bit"}

    r.close()          # the remaining measurements use their own contexts
    del flush
    torch.cuda.empty_cache()
    cpu = cpu_atrous = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, cores, sample = cpu_sample(scene, packed, 1, args.cpu_seconds, 8)
        cpu = {"value": v, "unit": "paths/s", "cores": cores, "kind": "port", "sample": sample}
        cpu_atrous = cpu_atrous_baseline()
    ttr = None
    if rank == 0 and world == 1 and not args.no_rmse and not mega:
        ttr = time_to_rmse(args)
    small = batch = None
    if rank == 0 and world == 1 and not args.no_extras and not mega:
        small = small_config()
        b = batch_measure(args, 0, 1, local, steps=2, warmup=3)
        batch = {k_: b[k_] for k_ in ("value", "unit", "ms_per_step", "view_done_ms", "view_finished_ms", "e2e",
                                      "rays_per_s", "autotune_table_ms", "autotune_kernels_table_ms")}
        batch["config"] = b["config"]
        batch["metric"] = b["metric"]

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "paths/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_s_max / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene generator)",
            "config": {"workload": "flagship 1920x1080, 8 bounces, 64 instances x 81,920-tri BLAS + 32 prims, "
                                   "2048x1024 RGBE env with importance sampling",
                       "step": f"one render call of {spp} samples per pixel ({paths_per_step:,} paths)",
                       "l2": "flushed between timed steps (256 MB write); path state and sample buffers exceed L2",
                       "parallelism": f"replicas x{world}", "render_mode": args.mode,
                       "path_pool": pool_paths,
                       "autotuned": None if tuned_k is None else {
                           "knobs": tuned_k["tuning"],
                           "trav_shape_names": {str(k_): v_ for k_, v_ in autotune_shapes().items()},
                           "table_ms": tuned_k["table"],
                           "method": "coordinate descent, one 64-spp call per candidate (CUDA events)"}},
            "rays_per_s": rays * world * args.steps / dev_s_max,
            "e2e": {"value": e2e_value, "unit": "paths/s", "h2d_bytes_per_step": 112,
                    "d2h_bytes_per_step": WIDTH * HEIGHT * 4},
            "gpu_launches": launches * args.steps,
            "stages": stages,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": achieved / peaks["hbm_gbs"],
                         "traffic": None if mega else EXTEND_DRAM_BYTES_PER_RAY * ext_rays_per_launch,
                         "dram_frac": None if mega or "k_wf_extend" not in stages else
                         EXTEND_DRAM_BYTES_PER_RAY * ext_rays_per_launch
                         / (stages["k_wf_extend"]["ms_total"] / 1e3 / stages["k_wf_extend"]["launches"])
                         / 1e9 / peaks["hbm_gbs"],
                         "traffic_source": None if mega else
                         "ncu dram__bytes_read.sum + dram__bytes_write.sum of steady-state k_wf_extend launches "
                         "of an 8,388,608-slot pool (mean of launches 13-15: 248 B per ray; a 2,097,152-slot pool "
                         "gives 250 B per ray), times this run's closest-hit rays per launch",
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                         else "fallback 6.65 TB/s",
                         "kernel": "k_render" if mega else KERNELS[dom],
                         "algorithmic_bytes_per_launch": bytes_per_launch,
                         "launch_ms": avg_launch_s * 1e3,
                         "note": "scene (~80 MB) is L2-resident; traversal is latency/divergence bound; stage "
                                 "times from a host-driven pass of the same kernels on the same stream",
                         "l2": {"peak": l2.value, "unit": "GB/s", "frac": achieved / l2.value,
                                "peak_source": "measured in this run: wgpt_probe_l2_read, a 64 MiB buffer read "
                                               "200 times with L2-only loads"}},
            "counters_per_step": {"paths": int(cnt[0]), "ext_rays": int(cnt[1]), "shadow_rays": int(cnt[2]),
                                  "nodes": int(cnt[3]), "tri_tests": int(cnt[5])},
            "clocks": clocks,
            "env_alias": env_alias,
        }
        if cpu:
            line["cpu_baseline"] = cpu
        if cpu_atrous:
            line["cpu_atrous_baseline"] = cpu_atrous
        if ttr:
            line["time_to_rmse"] = ttr
        if small:
            line["small_config"] = small
        if batch:
            line["batch"] = batch
        print(json.dumps(line), flush=True)
    from webgpuraytracer_b200 import replicas
    replicas.teardown(world)
    return 0


def scene_update_ms(r, rd, sc, scene, reps: int = 20) -> dict:
    """Host milliseconds per ABI call after one animation step of the scene (every primitive and
    instance moved, then re-packed by the caller): wgpt_update_objects (the updateObjects fast
    path: five small buffers and the TLAS node pairs), wgpt_update_scene (every buffer rewritten
    and validated) and wgpt_upload_scene (setScene).  Leaves the moved scene uploaded."""
    import ctypes as C
    for o in scene.objects:
        if o.type in ("Sphere", "Cube", "Cylinder", "Torus", "Model"):
            p = o.position
            o.set_position(float(p[0]) + 0.01, float(p[1]), float(p[2]))
    packed = sc.pack_scene_data(scene)      # keeps the buffers the descriptor points at alive
    desc = rd.scene_desc(packed)
    out = {}
    for name in ("wgpt_update_objects", "wgpt_update_scene", "wgpt_upload_scene"):
        fn = getattr(r.L, name)
        r._check(fn(r.ctx, C.byref(desc)), name)
        r.synchronize()
        t0 = time.perf_counter()
        for _ in range(reps):
            r._check(fn(r.ctx, C.byref(desc)), name)
        r.synchronize()
        out[name] = (time.perf_counter() - t0) / reps * 1e3
    out["note"] = "host wall time per call, the scene's packing excluded"
    return out


def run_batch(args):
    """--workload batch: 32 seeded views (sizes over 256^2..1920x1080, 4/16/64 spp, 8 bounces)
    of the 5.24 M-triangle scene.  The views are shared out over the ranks longest-first (LPT by
    width x height x spp; strong scaling of the fixed batch); each rank autotunes its path pool
    on a quarter-sample probe, then traces all its views in one render_views call per step and
    finishes every view with the learned denoiser.  Reports paths/s over all views and the
    p50/p99 of the per-view completion times (device clock from the start of the call's work to
    the view's last sample) and of the finished times (denoised image ready)."""
    rank, world, local = dist_setup(args.gpus)
    line = batch_measure(args, rank, world, local, args.steps, args.warmup)
    if rank == 0:
        print(json.dumps(line), flush=True)
    from webgpuraytracer_b200 import replicas
    replicas.teardown(world)
    return 0


def batch_measure(args, rank: int, world: int, local: int, steps: int, warmup: int) -> dict | None:
    """The batched-views measurement of run_batch; returns rank 0's line (None elsewhere)."""
    import torch
    from webgpuraytracer_b200 import autotune
    from webgpuraytracer_b200 import kpcn
    from webgpuraytracer_b200 import renderer as rd
    from webgpuraytracer_b200 import replicas
    from webgpuraytracer_b200 import scene as sc
    from webgpuraytracer_b200 import synth

    torch.cuda.set_device(local)
    scene = synth.batch_scene(1)
    packed = sc.pack_scene_data(scene)
    all_views = synth.batch_views(1, 32)
    work = [v["width"] * v["height"] * v["spp"] for v in all_views]
    mine = replicas.assign_lpt(work, world)[rank]
    views = [all_views[i] for i in mine]
    r = rd.Renderer(16, 16, device=local)
    r.set_scene(scene, packed=packed)
    r.set_views([(v["width"], v["height"]) for v in views])
    stream = torch.cuda.ExternalStream(r.stream_handle(), device=torch.device("cuda", local))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    spp = [v["spp"] for v in views]
    paths_mine = sum(v["width"] * v["height"] * v["spp"] for v in views)
    paths_all = sum(work)

    def params_for(step):
        ff = [step * 64] * len(views)
        return [synth.view_params(scene, packed, v, f, 1) for v, f in zip(views, ff)], ff

    def launch(step, timing=False):
        params, ff = params_for(step)
        return r.render_views(params, ff, spp, timing=timing)

    r.render_views_gbuffer(params_for(0)[0])
    probe_spp = [max(1, x // 4) for x in spp]
    p0, f0 = params_for(0)
    if args.pool:
        r.set_wavefront_config(args.pool, 1 << 30)
        tuned = {"pool_paths": args.pool, "units_per_pass": 1 << 30, "table": "fixed by --pool"}
    else:
        tuned = autotune.tune_wavefront(r, lambda: r.render_views(p0, f0, probe_spp, timing=False),
                                        units=(1 << 27, 1 << 30))
    tuned_k = autotune.tune_kernels(r, lambda: r.render_views(p0, f0, probe_spp, timing=False))
    net = kpcn.Kpcn(local, seed=1)   # untrained weights: the same kernels and cost as trained ones
    for i in range(len(views)):      # first use loads the network's kernels and sizes its buffers
        net.denoise_view(r, i)

    for i in range(warmup):
        launch(i)
    r.synchronize()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    sampler = ClockSampler(local)
    barrier(world)
    torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.3)
    for i in range(steps):
        with torch.cuda.stream(stream):
            flush.fill_(float(i))
            starts[i].record(stream)
        launch(warmup + i)
        with torch.cuda.stream(stream):
            ends[i].record(stream)
    r.synchronize()
    torch.cuda.synchronize()
    barrier(world)
    clocks = sampler.stop()
    dev_s = sum(s_.elapsed_time(e_) for s_, e_ in zip(starts, ends)) / 1e3
    dev_s_max = max_over_ranks(dev_s, world)
    value = paths_all * steps / dev_s_max
    # per-view completion (device stamps) and finishing by the learned denoiser, views in the
    # order their samples completed
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    done = launch(warmup + steps, timing=True)
    e1.record(stream)
    torch.cuda.synchronize()
    call_ms = e0.elapsed_time(e1)
    finished = [0.0] * len(views)
    t_acc = call_ms
    for i in sorted(range(len(views)), key=lambda j: done[j]):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        net.denoise_view(r, i)
        b.record(stream)
        torch.cuda.synchronize()
        t_acc += a.elapsed_time(b)
        finished[i] = t_acc
    done_all = replicas.gather_lists([float(x) for x in done], world)
    fin_all = replicas.gather_lists(finished, world)
    # end-to-end: params in, every view traced, denoised and read back as rgba8, every step
    outs = [np.empty((v["height"], v["width"], 4), np.uint8) for v in views]
    e2e_steps = max(1, min(steps, 4))
    barrier(world)
    t0 = time.perf_counter()
    for i in range(e2e_steps):
        launch(warmup + steps + 1 + i)
        for k_, o in enumerate(outs):
            net.denoise_view(r, k_)
            r._check(r.L.wgpt_read_view(r.ctx, k_, None, rd.ptr(o)), "read_view")
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    rep = stage_report(r, rd, lambda: launch(warmup), stream, flush, paths_mine, False)
    upd = scene_update_ms(r, rd, sc, scene)
    peaks, peak_kind = load_peaks()
    cnt = rep["cnt"]
    rays_all = replicas.sum_over_ranks(float(cnt[1] + cnt[2]), world)
    if rank == 0:
        line = {
            "metric": "paths/s, 32 batched views (uneven size and spp), 8 bounces", "value": value,
            "unit": "paths/s", "n_gpus": world, "steps": steps, "warmup": warmup,
            "ms_per_step": dev_s_max / steps * 1e3, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene and view generator)",
            "config": {"workload": "batched views: 32 views of 16 instances x 327,680-tri BLAS + 64 prims, "
                                   "2048x1024 RGBE env; sizes {256^2, 512^2, 1280x720, 1920x1080}, spp {4,16,64}",
                       "step": f"one render_views call per rank ({paths_all:,} paths over all ranks)",
                       "l2": "flushed between timed steps (256 MB write)",
                       "parallelism": f"views LPT-assigned over {world} rank(s)",
                       "autotuned": {"pool_paths": tuned["pool_paths"], "units_per_pass": tuned["units_per_pass"],
                                     **tuned_k["tuning"]}},
            "autotune_kernels_table_ms": tuned_k["table"],
            "autotune_table_ms": tuned["table"],
            "view_done_ms": {"p50": float(np.percentile(done_all, 50)), "p99": float(np.percentile(done_all, 99)),
                             "max": float(np.max(done_all))},
            "view_finished_ms": {"p50": float(np.percentile(fin_all, 50)), "p99": float(np.percentile(fin_all, 99)),
                                 "max": float(np.max(fin_all)),
                                 "note": "render call end + learned-denoiser passes in completion order"},
            "rays_per_s": rays_all * steps / dev_s_max,
            "scene_update_ms": upd,
            "e2e": {"value": paths_all * e2e_steps / e2e_s, "unit": "paths/s",
                    "h2d_bytes_per_step": 112 * len(all_views),
                    "d2h_bytes_per_step": sum(v["width"] * v["height"] * 4 for v in all_views),
                    "includes": "render, learned denoiser per view, rgba8 readback"},
            "gpu_launches": rep["launches"] * steps,
            "stages": rep["stages"],
            "roofline": {"bound": "hbm", "achieved": rep["achieved"], "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": rep["achieved"] / peaks["hbm_gbs"], "traffic": None,
                         "kernel": KERNELS[rep["dom"]], "launch_ms": rep["avg_launch_s"] * 1e3,
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"},
            "clocks": clocks,
        }
    net.close()
    r.close()
    return line if rank == 0 else None


def run_denoise(args):
    """--workload denoise: the learned denoiser's inference (1920x1080, untrained weights, which
    cost the same) and the a-trous filter (5 passes) on a 4-spp accumulation of the small-
    configuration scene; one step = one filter of the frame.  For kernel profiles."""
    import torch
    from webgpuraytracer_b200 import kpcn
    from webgpuraytracer_b200 import renderer as rd
    from webgpuraytracer_b200 import synth
    W, H = 1920, 1080
    scene = synth.small_scene(1, W, H, 4)
    scene.camera.aspect = W / H
    r = rd.Renderer(W, H, seed_fn=lambda: 7)
    r.set_scene(scene, isgbuf=True)
    r.render_gbuffer()
    r.reset()
    r.render(tsize=W, reps=4)
    k = kpcn.Kpcn(0, seed=1)
    st = torch.cuda.ExternalStream(r.stream_handle())
    atrous = rd.Denoiser(r, passes=5)
    res = {}
    for name, fn_ in (("kpcn", lambda: k.denoise(r, want_linear=False)), ("atrous", atrous.execute)):
        for _ in range(args.warmup):
            fn_()
        r.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(args.steps):
            fn_()
        e1.record(st)
        r.synchronize()
        torch.cuda.synchronize()
        res[name] = e0.elapsed_time(e1) / args.steps
    flops = kpcn.gemm_flops(W, H)
    peaks, kind = load_peaks()
    tf = flops / (res["kpcn"] / 1e3) / 1e12
    print(json.dumps({"metric": "denoise ms per 1920x1080 frame", "value": res["kpcn"], "unit": "ms",
                      "higher_is_better": False, "steps": args.steps, "warmup": args.warmup,
                      "atrous_ms": res["atrous"], "kpcn_gemm_tflops": tf,
                      "kpcn_frac_of_bf16_peak": tf / peaks.get("bf16_tflops", 1590.0),
                      "config": {"workload": "denoise 1920x1080, small-configuration scene at 4 spp"}}), flush=True)
    k.close()
    r.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--spp", type=int, default=SPP, help="samples per pixel per step (render call)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--mode", choices=["wavefront", "megakernel"], default="wavefront")
    ap.add_argument("--pool", type=int, default=0, help="wavefront path slots (0: library default)")
    ap.add_argument("--no-rmse", action="store_true", help="skip the time-to-RMSE measurement")
    ap.add_argument("--no-tune", action="store_true", help="keep the default kernel variants (no autotuning)")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the small-configuration and batched-views measurements of the default line")
    ap.add_argument("--rmse-threshold", type=float, default=0.01)
    ap.add_argument("--ref-spp", type=int, default=65536, help="samples of the FP64 reference image")
    ap.add_argument("--max-spp", type=int, default=4096, help="largest sample count of the RMSE sweep")
    ap.add_argument("--kpcn-scenes", type=int, default=64, help="flagship-family training scenes")
    ap.add_argument("--kpcn-crops", type=int, default=2, help="256x256 training windows per scene")
    ap.add_argument("--kpcn-target-spp", type=int, default=1024)
    ap.add_argument("--kpcn-steps", type=int, default=3000)
    ap.add_argument("--kpcn-spps", default="1,2,4,8,16,32,64", help="input samples per pixel of in-run training")
    ap.add_argument("--kpcn-schedule", default="0.65:1,0.2:0.3,0.15:0.1", help="lr phases of in-run training")
    ap.add_argument("--kpcn-weights", default="", help="trained weights (.npz; default: the package's flagship weights)")
    ap.add_argument("--kpcn-train", action="store_true", help="train the network in this run even if weights exist")
    ap.add_argument("--max-nn-spp", type=int, default=256, help="largest sample count the network is evaluated at")
    ap.add_argument("--workload", choices=["flagship", "batch", "denoise"], default="flagship",
                    help="flagship: 1080p 64 spp; batch: 32 uneven views of the 5.24 M-triangle scene; "
                         "denoise: learned and a-trous filters on one 1080p frame")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batch":
        return run_batch(args)
    if args.workload == "denoise":
        return run_denoise(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
