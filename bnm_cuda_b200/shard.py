"""Particle sharding over ranks (one process per GPU).

Particles of a generation are independent apart from the shared SC, noise
table and targets (the reference's run_simulations treats each particle
alone, bnm.cu:594-769), so a generation of ``n`` particles splits
into contiguous shards, one per rank, with no data-path collective.  The only
exchange is the one a host CMA-ES needs after the generation: every rank's
fit terms gathered, in particle order, on every rank.

``simulate`` is any callable (G, wEE, wEI) -> dict of per-particle arrays
(``Plan.run`` on the GPU; tests pass a stand-in on CPU ranks).
"""
from __future__ import annotations

import numpy as np

FIELDS = ("cost", "fic_penalty", "fc_corr", "fc_diff", "fcd_ks", "fic_ntrials", "fic_failed")


def shard_bounds(n: int, world: int, rank: int) -> tuple[int, int]:
    """[start, stop) of rank's contiguous shard of n particles; the first
    n % world ranks take one extra particle."""
    if world < 1 or not 0 <= rank < world or n < 0:
        raise ValueError("bad shard request")
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def gather(local: dict, n: int, fields=FIELDS) -> dict:
    """All-gather each field's local shard (variable length) into the full
    particle-ordered vector on every rank (torch.distributed, any backend)."""
    import torch
    import torch.distributed as dist

    world, rank = dist.get_world_size(), dist.get_rank()
    counts = [shard_bounds(n, world, r)[1] - shard_bounds(n, world, r)[0] for r in range(world)]
    width = max(counts)
    backend = dist.get_backend()
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    out = {}
    for f in fields:
        x = np.asarray(local[f], dtype=np.float64)
        if len(x) != counts[rank]:
            raise ValueError(f"{f}: rank {rank} holds {len(x)} values, its shard has {counts[rank]}")
        buf = torch.zeros(width, dtype=torch.float64, device=dev)
        buf[: len(x)] = torch.from_numpy(x).to(dev)
        parts = [torch.empty_like(buf) for _ in range(world)]
        dist.all_gather(parts, buf)
        out[f] = np.concatenate([p[:c].cpu().numpy() for p, c in zip(parts, counts)])
    return out


def run_sharded(simulate, G, wEE, wEI, fields=FIELDS) -> dict:
    """One generation over all ranks: this rank simulates its shard of the
    full parameter arrays, then every rank receives every particle's fields."""
    import torch.distributed as dist

    G = np.atleast_1d(G)
    n = len(G)
    a, b = shard_bounds(n, dist.get_world_size(), dist.get_rank())
    local = simulate(G[a:b], np.asarray(wEE)[a:b], np.asarray(wEI)[a:b]) if b > a else {f: np.zeros(0) for f in fields}
    return gather(local, n, fields)
