"""The N > 1 path on CPU: two gloo ranks each run their shard of an ensemble (replicas, no
exchange) through the oracle, with the barrier / max-over-ranks timing bench.py uses."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import tild_dist


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in ("gpu-tild_b200", "oracle", "tests"):
        sys.path.insert(0, os.path.join(root, p))
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    import time
    import oracle
    from helpers import small_diblock
    g = tild_dist.Group(backend="gloo", timeout_s=60)
    sizes = [60, 40, 30, 20, 20, 10]
    mine = tild_dist.shard(sizes, g.rank, g.world)
    g.barrier()
    t0 = time.perf_counter()
    done = 0
    for i in mine:
        s = small_diblock(3, 1, n_chains=sizes[i], N=5, seed=100 + i)
        o = oracle.Oracle(s)
        x, xo, nz = s.x.copy(), s.x.copy(), np.zeros_like(s.x)
        o.step(x, xo, nz, 1, True)
        done += s.ns
    dt = time.perf_counter() - t0
    tmax = g.max(dt)
    total = g.sum(done)
    out[rank] = (mine, dt, tmax, total)
    g.close()


def test_two_rank_ensemble_shards_and_reduces():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    shards = [out[r][0] for r in range(world)]
    assert sorted(shards[0] + shards[1]) == list(range(6)) and not set(shards[0]) & set(shards[1])
    assert out[0][2] == out[1][2] == pytest.approx(max(out[0][1], out[1][1]))
    assert out[0][3] == out[1][3] == sum([60, 40, 30, 20, 20, 10]) * 5


def test_shard_balances_particles():
    sizes = list(np.random.default_rng(0).integers(1000, 50000, size=256))
    loads = [sum(sizes[i] for i in tild_dist.shard(sizes, r, 8)) for r in range(8)]
    assert max(loads) / min(loads) < 1.05
