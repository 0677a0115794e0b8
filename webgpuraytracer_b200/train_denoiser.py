"""Builds the learned denoiser's training set at its stated scale and trains the network on it.

    python -m webgpuraytracer_b200.train_denoiser --out weights.npz
        [--family small|flagship] [--scenes 2000] [--first-seed 1000] [--crops 1]
        [--spps 1,2,4,8] [--target-spp 4096] [--target-f32]
        [--steps 40000] [--batch 16] [--crop 128] [--lr 1e-3] [--schedule 0.65:1,0.2:0.3,0.15:0.1]
        [--device 0] [--eval 16]

The set: for each seeded scene of the chosen family, `crops` 256x256 windows of its view,
progressive inputs at each sample count of --spps (one example each) and a target at
--target-spp with an independent sample stream accumulated in FP64 (FP32 running mean with
--target-f32), all path traced on the GPU by this renderer.  The defaults are the learned-denoiser configuration: 2,000 scenes of the
small-configuration family, 256x256, 1/2/4/8-spp inputs, 4096-spp targets (the set is held in
device memory: about 5 MB an example, 40 GB for the 8,000 examples).  The flagship family
(seeded 8-bounce flagship scenes with their own cameras, windows of their 1920x1080 views)
trains the weights used at the flagship's resolution.  The network is then trained by the
project's own forward/backward/Adam kernels (wgpt_kpcn_train) on random crop x crop crops; the
learning rate is --lr times the factor of each --schedule phase (fraction of the steps:factor).
Its FP32 parameters and the recipe are written to --out (kpcn.load_weights reads them).  With
--eval N the script also reports the display-space RMSE of the noisy input, the a-trous filter
and the network on N held-out scenes (seeds above the training range).
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np


def parse_schedule(text: str, steps: int) -> list[tuple[int, float]]:
    """'0.65:1,0.2:0.3,0.15:0.1' -> [(steps of the phase, lr factor)], the last phase taking the
    remainder so the phases sum to `steps`."""
    phases = []
    for part in text.split(","):
        frac, factor = part.split(":")
        phases.append((float(frac), float(factor)))
    out, used = [], 0
    for i, (frac, factor) in enumerate(phases):
        n = steps - used if i == len(phases) - 1 else min(int(steps * frac + 0.5), steps - used)
        out.append((max(n, 0), factor))
        used += n
    return [(n, f) for n, f in out if n > 0]


def train(k, steps: int, batch: int, crop: int, lr: float, schedule: str, seed: int = 1) -> np.ndarray:
    """Adam steps over the phases of `schedule`; returns every step's loss."""
    losses = []
    for i, (n, factor) in enumerate(parse_schedule(schedule, steps)):
        losses.append(k.train(n, batch=batch, crop=crop, lr=lr * factor, seed=seed + 7919 * i))
    return np.concatenate(losses) if losses else np.zeros(0, np.float32)


def evaluate(k, family: str, seeds, size: int = 256, spp: int = 4, target_spp: int = 4096) -> dict:
    """Display RMSE (mean over scenes) of noisy input, a-trous (5 passes) and network."""
    from . import kpcn, synth
    from . import renderer as rd
    res = {"noisy": [], "atrous_5": [], "kpcn": []}
    for seed in seeds:
        if family == "small":
            s = synth.small_scene(int(seed), size, size, 4)
            s.camera.aspect = 1.0
            w = h = size
        else:
            s = kpcn.flagship_family_scene(int(seed))
            w, h = 1920, 1080
        t = rd.Renderer(w, h, seed_fn=lambda: 300_000 + int(seed))
        t.set_scene(s)
        t.render(tsize=max(w, h), reps=target_spp)
        target = t.read_accum()
        t.close()
        r = rd.Renderer(w, h, seed_fn=lambda: int(seed))
        r.set_scene(s, isgbuf=True)
        r.render_gbuffer()
        r.reset()
        r.render(tsize=max(w, h), reps=spp)
        res["noisy"].append(kpcn.rmse(r.read_accum(), target))
        dn = rd.Denoiser(r, passes=5)
        dn.execute()
        comp = dn.read()[1]
        res["atrous_5"].append(float(np.sqrt(np.mean((np.clip(comp[..., :3], 0, 1) - kpcn.tonemap(target)) ** 2))))
        res["kpcn"].append(kpcn.rmse(k.denoise(r), target))
        r.close()
    return {m: float(np.mean(v)) for m, v in res.items()}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--out", required=True, help="where to write the trained parameters and recipe (.npz)")
    ap.add_argument("--family", choices=["small", "flagship"], default="small")
    ap.add_argument("--scenes", type=int, default=2000)
    ap.add_argument("--first-seed", type=int, default=1000)
    ap.add_argument("--crops", type=int, default=1, help="256x256 windows per flagship-family scene")
    ap.add_argument("--spps", default="1,2,4,8", help="input samples per pixel, comma-separated")
    ap.add_argument("--target-spp", type=int, default=4096)
    ap.add_argument("--target-f32", action="store_true", help="targets as the FP32 running mean")
    ap.add_argument("--steps", type=int, default=40000)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--crop", type=int, default=128)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--schedule", default="1:1", help="phases fraction:lr-factor, comma-separated")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--eval", type=int, default=0, help="held-out scenes to evaluate on afterwards")
    args = ap.parse_args(argv)
    from . import kpcn
    spps = tuple(int(v) for v in args.spps.split(","))
    k = kpcn.Kpcn(args.device, seed=1)
    seeds = range(args.first_seed, args.first_seed + args.scenes)
    t0 = time.perf_counter()
    if args.family == "small":
        n = kpcn.build_training_set(k, seeds, 256, spps, args.target_spp, device=args.device,
                                    target_f64=not args.target_f32)
    else:
        n = kpcn.build_flagship_training_set(k, seeds, crops=args.crops, spps=spps, target_spp=args.target_spp,
                                             device=args.device, target_f64=not args.target_f32)
    t_data = time.perf_counter() - t0
    t0 = time.perf_counter()
    losses = train(k, args.steps, args.batch, args.crop, args.lr, args.schedule)
    t_train = time.perf_counter() - t0
    report = {"family": args.family, "scenes": args.scenes, "first_seed": args.first_seed, "crops": args.crops,
              "examples": n, "input_spp": list(spps), "target_spp": args.target_spp,
              "target_accumulation": "fp32" if args.target_f32 else "fp64", "steps": args.steps,
              "batch": args.batch, "crop": args.crop, "lr": args.lr, "schedule": args.schedule,
              "data_s": t_data, "train_s": t_train,
              "loss_first_100": float(losses[:100].mean()), "loss_last_500": float(losses[-500:].mean()),
              "command": "python -m webgpuraytracer_b200.train_denoiser " + " ".join(sys.argv[1:] if argv is None
                                                                                    else argv)}
    if args.eval:
        ev_seeds = range(args.first_seed + args.scenes + 1000, args.first_seed + args.scenes + 1000 + args.eval)
        report["held_out_4spp"] = evaluate(k, args.family, ev_seeds)
    kpcn.save_weights(k, args.out, report)
    print(json.dumps(report), flush=True)
    k.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
