"""Particle sharding over ranks (bnm_cuda_b200.shard) as world-size-2 gloo
process groups on CPU: contiguous shards cover every particle once, and the
all-gather returns every rank the full particle-ordered fit terms, equal to a
single-process run.  The per-particle stand-in for the simulator is a
deterministic function of the particle's parameters (no GPU on CPU ranks)."""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

from bnm_cuda_b200 import shard


def fake_simulate(G, wEE, wEI):
    G, wEE, wEI = np.asarray(G), np.asarray(wEE), np.asarray(wEI)
    c = np.sin(3 * G) + wEE.mean(1) ** 2 - wEI.mean(1)
    return {"cost": c, "fic_penalty": 0.1 * G, "fc_corr": np.cos(G), "fc_diff": wEE[:, 0], "fcd_ks": wEI[:, 0],
            "fic_ntrials": (G * 3).astype(int), "fic_failed": (G > 3).astype(int)}


@pytest.mark.parametrize("n,world", [(10, 2), (7, 2), (1, 2), (0, 3), (256, 8), (5, 8)])
def test_shard_bounds_partition(n, world):
    spans = [shard.shard_bounds(n, world, r) for r in range(world)]
    assert spans[0][0] == 0 and spans[-1][1] == n
    for (a, b), (c, d) in zip(spans, spans[1:]):
        assert b == c and b - a >= d - c >= b - a - 1


def test_shard_bounds_rejects_bad_requests():
    for args in [(4, 0, 0), (4, 2, 2), (-1, 2, 0)]:
        with pytest.raises(ValueError):
            shard.shard_bounds(*args)


def _rank(rank, world, port, n, q):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(0)
        G, wEE, wEI = rng.uniform(0.5, 4, n), rng.uniform(0.05, 0.75, (n, 6)), rng.uniform(0.05, 0.75, (n, 6))
        out = shard.run_sharded(fake_simulate, G, wEE, wEI)
        q.put((rank, {k: v.tolist() for k, v in out.items()}))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("n", [9, 64])
def test_run_sharded_gathers_every_particle_on_every_rank(n):
    ctx = mp.get_context("spawn")
    q, port, world = ctx.Queue(), _free_port(), 2
    procs = [ctx.Process(target=_rank, args=(r, world, port, n, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    rng = np.random.default_rng(0)
    G, wEE, wEI = rng.uniform(0.5, 4, n), rng.uniform(0.05, 0.75, (n, 6)), rng.uniform(0.05, 0.75, (n, 6))
    want = fake_simulate(G, wEE, wEI)
    for r in range(world):
        for k in shard.FIELDS:
            np.testing.assert_allclose(got[r][k], want[k], rtol=0, atol=0, err_msg=(r, k))
