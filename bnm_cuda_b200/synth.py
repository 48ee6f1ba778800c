"""Seeded synthetic inputs and the benchmark workloads.

The reference ships one example connectome (example/input/SC.txt, 100 nodes)
and no benchmark data.  The workloads below are defined by their shapes and
value distributions and generated from fixed seeds:

* structural connectome: symmetric, zero diagonal, Bernoulli(density) on the
  upper triangle, log-normal(mu=0, sigma=1) weights, scaled so that the
  largest row sum is 1 (``numpy.random.default_rng(seed)``);
* CMA-ES-style particles: G, wEE, wEI uniform on the given bounds.

Window and frame bookkeeping follows run_CMAES.cpp:476-594 (frames =
T / TR + 1, n_vols_remove = BNM_BOLD_REMOVE * 1000 / TR, FCD windows
centred from ws/2 to corr_len-1-ws/2 in steps of ``window_step``).
"""
from __future__ import annotations

import dataclasses
import numpy as np


def make_sc(n: int, density: float, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    iu = np.triu_indices(n, 1)
    mask = rng.random(iu[0].size) < density
    w = rng.lognormal(mean=0.0, sigma=1.0, size=iu[0].size) * mask
    sc = np.zeros((n, n))
    sc[iu] = w
    sc = sc + sc.T
    rs = sc.sum(1).max()
    if rs > 0:
        sc /= rs
    return sc


def uniform_params(n_sims: int, n_nodes: int, seed: int, g=(0.5, 4.0), wee=(0.05, 0.75), wei=(0.05, 0.75)):
    """Homogeneous particles: G [n], wEE / wEI [n, N] (same value on every node)."""
    rng = np.random.default_rng(seed)
    G = rng.uniform(*g, size=n_sims)
    we = rng.uniform(*wee, size=n_sims)
    wi = rng.uniform(*wei, size=n_sims)
    return G, np.repeat(we[:, None], n_nodes, 1), np.repeat(wi[:, None], n_nodes, 1)


def n_pairs(n: int, exc_interhem: bool) -> int:
    """check_fit.cpp:24-32 / run_CMAES.cpp:494-500."""
    p = n * (n - 1) // 2
    if exc_interhem:
        p -= (n // 2) ** 2
    return p


def windows(corr_len: int, window_size: int, window_step: int):
    """Inclusive (start, end) frame indices relative to the first kept frame
    (check_fit.cpp:79-106; run_CMAES.cpp:531-556 adds n_vols_remove)."""
    first, last = window_size // 2, corr_len - 1 - window_size // 2
    out = []
    c = first
    while c <= last:
        s, e = max(c - window_size // 2, 0), min(c + window_size // 2, corr_len - 1)
        out.append((s, e))
        c += window_step
    return out


@dataclasses.dataclass
class Workload:
    name: str
    nodes: int
    n_sims: int
    time_steps: int  # ms
    bold_tr: int  # ms
    window_size: int
    window_step: int
    bold_remove_s: int = 30
    exc_interhem: bool = True
    sc_density: float = 0.3
    sc_seed: int = 0
    noise_seed: int = 410
    param_seed: int = 1

    @property
    def frames(self) -> int:
        return self.time_steps // self.bold_tr + 1

    @property
    def n_vols_remove(self) -> int:
        return self.bold_remove_s * 1000 // self.bold_tr

    @property
    def corr_len(self) -> int:
        return self.frames - self.n_vols_remove

    @property
    def n_windows(self) -> int:
        return len(windows(self.corr_len, self.window_size, self.window_step))

    @property
    def n_pairs(self) -> int:
        return n_pairs(self.nodes, self.exc_interhem)

    def substeps(self, fic_restarts: int = 0, sampling_end: int = 10000) -> int:
        return 10 * (self.time_steps + 1) + 10 * sampling_end * fic_restarts


# Single FP64-checkable simulation (60 s kept after a 5 s transient).
CONFIG0 = Workload("single-N100-65s", nodes=100, n_sims=1, time_steps=65_000, bold_tr=1000, window_size=10,
                   window_step=2, bold_remove_s=5)
# One CMA-ES generation: 256 particles, N=100, 450 s at TR 0.72 s, window 44 step 1.
CONFIG1 = Workload("cmaes-generation-N100-450s-x256", nodes=100, n_sims=256, time_steps=450_000, bold_tr=720,
                   window_size=44, window_step=1)
# Precision stress: 64 particles, N=400 (10 % density), 600 s at TR 0.5 s, all pairs kept.
CONFIG2 = Workload("fcd-precision-N400-600s-x64", nodes=400, n_sims=64, time_steps=600_000, bold_tr=500,
                   window_size=44, window_step=1, bold_remove_s=0, exc_interhem=False, sc_density=0.1)
