"""Surrogate-screened CMA-ES (no counterpart in the reference).

A small MLP, trained on the device by the library's own kernels
(``bnm_mlp_*``: BF16 tensor-core GEMMs with FP32 accumulation, Adam), maps
    (G, wEE, wEI) scaled to [0, 1]  +  a 16-value SC spectral summary
to the fit terms of a simulation (FC correlation, FC mean difference, FCD KS
distance, FIC penalty).  Screened CMA-ES draws ``oversample`` x lambda
candidates per generation from the current search distribution, ranks them
by predicted cost and injects the best lambda as the generation's samples;
only simulated costs reach the optimiser.  Every reported fit is a simulated
one.  Screening uses only the ranking of candidates, so the surrogate is
trusted when it ranks held-out simulations well (Spearman correlation of
predicted and simulated cost at least ``min_rank_corr``) and screening is
switched off (plain CMA-ES) otherwise, or once its error on the simulated
candidates exceeds their spread two generations running.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import time

import numpy as np

from . import CMAES, Config, Plan, _check, _ptr, lib

N_SPECTRAL = 16
OUTPUTS = ("fc_corr", "fc_diff", "fcd_ks", "fic_penalty")


def spectral_summary(sc: np.ndarray, k: int = N_SPECTRAL) -> np.ndarray:
    """The k smallest non-zero eigenvalues of the normalised graph Laplacian
    I - D^-1/2 SC D^-1/2 (zero-padded when the graph is smaller)."""
    d = sc.sum(1)
    inv = np.where(d > 0, 1.0 / np.sqrt(np.maximum(d, 1e-300)), 0.0)
    L = np.eye(len(sc)) - inv[:, None] * sc * inv[None, :]
    ev = np.sort(np.linalg.eigvalsh((L + L.T) / 2))
    ev = ev[ev > 1e-9][:k]
    return np.pad(ev, (0, k - len(ev)))


@dataclasses.dataclass
class Bounds:
    G: tuple = (0.5, 4.0)
    wEE: tuple = (0.05, 0.75)
    wEI: tuple = (0.05, 0.75)

    def to_params(self, x01: np.ndarray):
        """x01 [3][n] in [0, 1] -> G [n], wEE [n], wEI [n]."""
        lo = np.array([self.G[0], self.wEE[0], self.wEI[0]])[:, None]
        hi = np.array([self.G[1], self.wEE[1], self.wEI[1]])[:, None]
        p = lo + (hi - lo) * x01
        return p[0], p[1], p[2]


def features(x01: np.ndarray, spec: np.ndarray) -> np.ndarray:
    """x01 [3][n] -> [n][3 + len(spec)] float32."""
    n = x01.shape[1]
    return np.hstack([x01.T, np.repeat(spec[None, :], n, 0)]).astype(np.float32)


def simulate(plan: Plan, x01: np.ndarray, bounds: Bounds, batch: int | None = None) -> np.ndarray:
    """Runs the plain path on every column of x01; returns [n][4] fit terms."""
    G, we, wi = bounds.to_params(x01)
    n, N = len(G), plan.cfg.nodes
    batch = batch or plan.cfg.max_sims
    out = np.zeros((n, len(OUTPUTS)))
    for s in range(0, n, batch):
        e = min(n, s + batch)
        r = plan.run(G[s:e], np.repeat(we[s:e, None], N, 1), np.repeat(wi[s:e, None], N, 1), outputs=())
        out[s:e] = np.stack([r[k] for k in OUTPUTS], 1)
    return out


def cost_of(terms: np.ndarray, use_fc_diff: bool = True) -> np.ndarray:
    """Total fit cost (what CMA-ES minimises): 1 - r_FC (+ |dmean|) + KS + FIC penalty."""
    c = 1.0 - terms[:, 0] + terms[:, 2] + terms[:, 3]
    if use_fc_diff:
        c = c + terms[:, 1]
    return c


class MLP:
    """The device MLP (bnm_mlp_*), with input / target standardisation."""

    def __init__(self, in_dim: int, out_dim: int = len(OUTPUTS), hidden: int = 256, layers: int = 4,
                 max_batch: int = 1024, seed: int = 0, device: int = 0):
        L = lib()
        L.bnm_mlp_create.argtypes = [C.c_int32] * 5 + [C.c_uint64, C.c_int32, C.POINTER(C.c_void_p)]
        L.bnm_mlp_destroy.argtypes = [C.c_void_p]
        L.bnm_mlp_num_params.argtypes = [C.c_void_p]
        L.bnm_mlp_num_params.restype = C.c_int64
        L.bnm_mlp_get_params.argtypes = [C.c_void_p, C.c_void_p]
        L.bnm_mlp_set_params.argtypes = [C.c_void_p, C.c_void_p]
        L.bnm_mlp_train.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_float,
                                    C.c_uint64, C.c_void_p]
        L.bnm_mlp_predict.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]
        L.bnm_mlp_loss_and_grads.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]
        h = C.c_void_p()
        _check(L.bnm_mlp_create(in_dim, hidden, layers, out_dim, max_batch, seed, device, C.byref(h)))
        self._h, self.in_dim, self.out_dim, self.hidden, self.layers = h, in_dim, out_dim, hidden, layers
        self.max_batch = max_batch
        self.x_mu = np.zeros(in_dim, np.float32)
        self.x_sd = np.ones(in_dim, np.float32)
        self.y_mu = np.zeros(out_dim, np.float32)
        self.y_sd = np.ones(out_dim, np.float32)

    def close(self):
        if getattr(self, "_h", None):
            lib().bnm_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def n_params(self) -> int:
        return lib().bnm_mlp_num_params(self._h)

    def get_params(self) -> np.ndarray:
        out = np.zeros(self.n_params, np.float32)
        _check(lib().bnm_mlp_get_params(self._h, _ptr(out)))
        return out

    def set_params(self, flat: np.ndarray):
        flat = np.ascontiguousarray(flat, np.float32)
        _check(lib().bnm_mlp_set_params(self._h, _ptr(flat)))

    def loss_and_grads(self, X: np.ndarray, Y: np.ndarray):
        """Raw (already normalised) batch -> (loss, flat gradient)."""
        X = np.ascontiguousarray(X, np.float32)
        Y = np.ascontiguousarray(Y, np.float32)
        loss = C.c_float()
        g = np.zeros(self.n_params, np.float32)
        _check(lib().bnm_mlp_loss_and_grads(self._h, _ptr(X), _ptr(Y), len(X), C.byref(loss), _ptr(g)))
        return loss.value, g

    def fit(self, X: np.ndarray, Y: np.ndarray, epochs: int = 60, batch: int = 256, lr: float = 1e-3,
            seed: int = 0) -> np.ndarray:
        self.x_mu, self.x_sd = X.mean(0).astype(np.float32), (X.std(0) + 1e-6).astype(np.float32)
        self.y_mu, self.y_sd = Y.mean(0).astype(np.float32), (Y.std(0) + 1e-6).astype(np.float32)
        Xn = np.ascontiguousarray((X - self.x_mu) / self.x_sd, np.float32)
        Yn = np.ascontiguousarray((Y - self.y_mu) / self.y_sd, np.float32)
        losses = np.zeros(epochs, np.float32)
        _check(lib().bnm_mlp_train(self._h, _ptr(Xn), _ptr(Yn), len(Xn), epochs, min(batch, len(Xn)), lr, seed,
                                   _ptr(losses)))
        return losses

    def fine_tune(self, X: np.ndarray, Y: np.ndarray, epochs: int = 4, batch: int = 64, lr: float = 3e-4,
                  seed: int = 0) -> np.ndarray:
        """More training on new data with the normalisation of the first fit."""
        Xn = np.ascontiguousarray((X - self.x_mu) / self.x_sd, np.float32)
        Yn = np.ascontiguousarray((Y - self.y_mu) / self.y_sd, np.float32)
        losses = np.zeros(epochs, np.float32)
        _check(lib().bnm_mlp_train(self._h, _ptr(Xn), _ptr(Yn), len(Xn), epochs, min(batch, len(Xn)), lr, seed,
                                   _ptr(losses)))
        return losses

    def predict(self, X: np.ndarray) -> np.ndarray:
        Xn = np.ascontiguousarray((X - self.x_mu) / self.x_sd, np.float32)
        out = np.zeros((len(Xn), self.out_dim), np.float32)
        _check(lib().bnm_mlp_predict(self._h, _ptr(Xn), len(Xn), _ptr(out)))
        return out * self.y_sd + self.y_mu


def train_surrogate(plan: Plan, bounds: Bounds, spec: np.ndarray, n_train: int, seed: int = 0, epochs: int = 60,
                    holdout: float = 0.1, batch: int = 256, lr: float = 1e-3):
    """Simulates n_train uniform parameter sets, trains the MLP, and reports the
    held-out RMSE of the predicted cost.  Returns (mlp, info)."""
    rng = np.random.default_rng(seed)
    x01 = rng.random((3, n_train))
    t0 = time.perf_counter()
    terms = simulate(plan, x01, bounds)
    t_sim = time.perf_counter() - t0
    X, Y = features(x01, spec), terms.astype(np.float32)
    n_val = max(1, int(holdout * n_train))
    mlp = MLP(X.shape[1], Y.shape[1], seed=seed)
    mlp.train_X, mlp.train_Y = X[n_val:], Y[n_val:]  # kept for replay during online fine-tuning
    t1 = time.perf_counter()
    losses = mlp.fit(X[n_val:], Y[n_val:], epochs=epochs, batch=batch, lr=lr, seed=seed)
    t_fit = time.perf_counter() - t1
    pred = mlp.predict(X[:n_val])
    true_cost, pred_cost = cost_of(terms[:n_val]), cost_of(pred.astype(np.float64))
    rmse = float(np.sqrt(np.mean((true_cost - pred_cost) ** 2)))
    from scipy.stats import spearmanr

    rho = float(spearmanr(true_cost, pred_cost).correlation)
    return mlp, dict(n_train=n_train, sim_s=t_sim, fit_s=t_fit, final_loss=float(losses[-1]), holdout_rmse=rmse,
                     holdout_spearman=rho, losses=losses.tolist())


def run_cmaes(plan: Plan, bounds: Bounds, lam: int, generations: int, seed: int, mlp: MLP | None = None,
              spec: np.ndarray | None = None, oversample: int = 8, min_rank_corr: float = 0.9,
              holdout_spearman: float | None = None, cand_seed: int = 12345, replay: int = 1024):
    """Plain CMA-ES, or surrogate-pre-screened CMA-ES when an MLP is given and
    its held-out rank correlation is at least ``min_rank_corr``.

    Screening: each generation draws oversample*lambda candidates from the
    current N(m, sigma^2 C), keeps the lambda with the lowest predicted cost,
    injects them as the generation's samples (bnm_cmaes_set_samples) and
    simulates them, so CMA-ES only ever sees simulated costs.  The surrogate
    is then fine-tuned on everything simulated so far (plus a replay of its
    training set), which makes it accurate where the search is.  Screening
    stops for good once the surrogate no longer separates the candidates: its
    error on the simulated ones exceeds their spread two generations in a
    row.  Returns the best simulated cost and wall time per generation."""
    screened = mlp is not None and (holdout_spearman is None or holdout_spearman >= min_rank_corr)
    es = CMAES(lam, 3, seed, generations + 1, from_env=False)
    rng = np.random.default_rng(cand_seed)
    best, best_x, hist, walls, errs, spreads, bad = np.inf, None, [], [], [], [], 0
    seen_X, seen_Y = [], []
    screened_gens = 0
    t0 = time.perf_counter()
    for gen in range(generations):
        if screened:
            m, sigma, Cm = es.state()
            cov = sigma * sigma * (Cm + Cm.T) / 2
            cand = rng.multivariate_normal(m, cov, size=oversample * lam, method="cholesky").T
            pred = cost_of(mlp.predict(features(np.clip(cand, 0.0, 1.0), spec)).astype(np.float64))
            top = np.argsort(pred)[:lam]
            es.set_samples(cand[:, top])
        feas, _, _ = es.samples()
        terms = simulate(plan, feas, bounds)
        cost = cost_of(terms)
        if screened:
            screened_gens += 1
            errs.append(float(np.sqrt(np.mean((pred[top] - cost) ** 2))))
            spreads.append(float(np.std(cost)))
            bad = bad + 1 if errs[-1] > spreads[-1] else 0
            seen_X.append(features(feas, spec))
            seen_Y.append(terms.astype(np.float32))
            if bad >= 2:
                screened = False
            else:
                k = min(replay, len(mlp.train_X))
                ridx = rng.choice(len(mlp.train_X), size=k, replace=False)
                mlp.fine_tune(np.vstack(seen_X + [mlp.train_X[ridx]]), np.vstack(seen_Y + [mlp.train_Y[ridx]]),
                              epochs=4, batch=64, seed=gen)
        k = int(np.argmin(cost))
        if cost[k] < best:
            best, best_x = float(cost[k]), feas[:, k].copy()
        hist.append(best)
        walls.append(time.perf_counter() - t0)
        if es.tell(cost)[0] >= es.it_max:
            break
    return dict(screened=mlp is not None, screened_generations=screened_gens, best=best,
                best_x=None if best_x is None else best_x.tolist(), best_hist=hist, wall_hist=walls,
                online_rmse=errs, candidate_spread=spreads, simulations=len(hist) * lam)


def time_to_fit(screen: dict, plain: dict, tol: float = 0.01):
    """Wall time the screened run needs to come within tol of the plain run's
    final best, and its ratio to the plain run's total wall time."""
    target = plain["best"] + tol
    for b, w in zip(screen["best_hist"], screen["wall_hist"]):
        if b <= target:
            return w, w / plain["wall_hist"][-1]
    return None, None
