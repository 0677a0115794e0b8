"""Data-parallel training's host logic on two gloo ranks (CPU).

kpcn.train_data_parallel drives any model with the learned denoiser's training interface
(n_params, get/set_params, grads into a buffer, apply(buffer, scale, lr)).  Here a small
least-squares model stands in for the network: each rank holds different examples and draws
its own batches; after every step both ranks must hold identical weights, equal to a single
process that averages the two ranks' gradients and takes the same Adam steps.
"""
from __future__ import annotations

import os
import socket

import numpy as np
import torch
import torch.multiprocessing as mp

from webgpuraytracer_b200 import kpcn

DIM, STEPS, BATCH, LR = 6, 25, 4, 0.05


class LstsqModel:
    """p . x ~ y over this rank's examples; Adam with the network's constants."""

    def __init__(self, rank: int, init_seed: int):
        rng = np.random.default_rng(100 + rank)
        self.x = rng.normal(size=(32, DIM))
        self.y = self.x @ np.linspace(-1, 1, DIM) + 0.1 * rng.normal(size=32)
        self.p = np.random.default_rng(init_seed).normal(size=DIM).astype(np.float32)
        self.n_params = DIM
        self.m = np.zeros(DIM)
        self.v = np.zeros(DIM)
        self.t = 0

    def get_params(self):
        return self.p.copy()

    def set_params(self, a):
        self.p = np.asarray(a, np.float32).copy()
        self.m[:] = 0
        self.v[:] = 0
        self.t = 0

    def batch_grad(self, batch, seed):
        idx = np.random.default_rng(seed).integers(0, len(self.x), batch)
        r = self.x[idx] @ self.p - self.y[idx]
        return float(np.mean(r * r)), (2.0 * (r[:, None] * self.x[idx]).mean(0)).astype(np.float32)

    def grads(self, batch, crop, seed, buf):
        loss, g = self.batch_grad(batch, seed)
        buf.copy_(torch.from_numpy(g))
        return loss

    def apply(self, buf, scale, lr):
        g = buf.numpy().astype(np.float64) * scale
        self.t += 1
        self.m = 0.9 * self.m + 0.1 * g
        self.v = 0.999 * self.v + 0.001 * g * g
        mh = self.m / (1 - 0.9 ** self.t)
        vh = self.v / (1 - 0.999 ** self.t)
        self.p = (self.p - lr * mh / (np.sqrt(vh) + 1e-8)).astype(np.float32)


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank: int, world: int, port: int, out):
    import torch.distributed as dist
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "MASTER_ADDR": "127.0.0.1",
                       "MASTER_PORT": str(port)})
    dist.init_process_group("gloo", rank=rank, world_size=world)
    model = LstsqModel(rank, init_seed=7 + rank)      # different initial weights: rank 0's win
    losses = kpcn.train_data_parallel(model, STEPS, batch=BATCH, crop=16, lr=LR, seed=3, device="cpu")
    out.put((rank, model.get_params(), losses))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_data_parallel_training_matches_averaged_gradients():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert np.array_equal(res[0][1], res[1][1])          # identical weights on every rank
    assert np.array_equal(res[0][2], res[1][2])          # the same (rank-averaged) loss curve
    # single-process reference: rank 0's initial weights, the two ranks' batches averaged
    models = [LstsqModel(r, init_seed=7) for r in range(world)]
    ref = LstsqModel(0, init_seed=7)
    for step in range(STEPS):
        gs = [m.batch_grad(BATCH, (3 * 1_000_003 + step) * world + r)[1] for r, m in enumerate(models)]
        total = torch.from_numpy(gs[0] + gs[1])
        ref.apply(total, 1.0 / world, LR)
        for m in models:
            m.p = ref.p.copy()
    np.testing.assert_allclose(res[0][1], ref.p, rtol=1e-6, atol=1e-6)
    assert res[0][2][-1] < res[0][2][0]                  # training reduces the loss
