"""Replicated rendering's host logic on two gloo ranks (CPU): the job time is the slowest
rank's, per-rank seeds differ, and merging running means equals the mean of all samples."""
from __future__ import annotations

import os
import socket

import numpy as np
import torch.multiprocessing as mp

from webgpuraytracer_b200 import replicas


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank: int, world: int, port: int, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    r, w, _ = replicas.setup("gloo", timeout_s=60)
    assert (r, w) == (rank, world)
    t = replicas.max_over_ranks(1.5 + rank, w)
    tot = replicas.sum_over_ranks(10 * (rank + 1), w)
    rng = np.random.default_rng(rank)
    samples = 3 + rank                      # ranks may have rendered different sample counts
    acc = rng.random((4, 5, 4))
    merged, n = replicas.merge_accumulations(acc, samples, w)
    replicas.barrier(w)
    out.put((rank, t, tot, replicas.rank_seed(1, rank), acc, samples, merged, n))
    replicas.teardown(w)


def test_two_gloo_ranks():
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
    assert all(r[1] == 2.5 for r in res)                 # max over ranks
    assert all(r[2] == 30.0 for r in res)                # sum over ranks
    assert res[0][3] != res[1][3]                        # distinct sample streams
    expect = (res[0][4] * res[0][5] + res[1][4] * res[1][5]) / (res[0][5] + res[1][5])
    for r in res:
        np.testing.assert_allclose(r[6], expect, rtol=1e-12)
        assert r[7] == res[0][5] + res[1][5]


def test_single_process_defaults():
    assert replicas.max_over_ranks(3.0, 1) == 3.0
    a = np.ones((2, 2, 4))
    m, n = replicas.merge_accumulations(a, 5, 1)
    assert m is a and n == 5


def test_lpt_assignment_balances_views():
    from webgpuraytracer_b200 import synth
    views = synth.batch_views(1, 32)
    work = [v["width"] * v["height"] * v["spp"] for v in views]
    for world in (1, 2, 4, 8):
        parts = replicas.assign_lpt(work, world)
        assert sorted(i for p in parts for i in p) == list(range(32))
        loads = [sum(work[i] for i in p) for p in parts]
        # LPT is within 4/3 of optimal; the optimum is at least max(total/world, largest job)
        bound = max(sum(work) / world, max(work))
        assert max(loads) <= bound * 4 / 3 + 1
    assert replicas.assign_lpt([5, 4, 3, 3, 3], 2) == [[0, 3], [1, 2, 4]]
