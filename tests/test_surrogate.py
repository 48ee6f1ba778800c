"""MLP surrogate: device gradients against the FP64 oracle, training, and what
pre-screening gains over picking candidates without it (GPU)."""
import numpy as np
import pytest

import bnm_cuda_b200 as B
from bnm_cuda_b200 import surrogate as S
from bnm_cuda_b200 import synth


def test_spectral_summary_cpu():
    sc = synth.make_sc(20, 0.5, 1)
    s = S.spectral_summary(sc)
    assert s.shape == (16,) and np.all(np.diff(s) >= -1e-12) and s[0] > 0
    d = sc.sum(1)
    L = np.eye(20) - sc / np.sqrt(np.outer(d, d))
    np.testing.assert_allclose(s, np.sort(np.linalg.eigvalsh(L))[1:17], atol=1e-12)


@pytest.mark.gpu
def test_mlp_gradients_match_fp64_oracle():
    from oracle import mlp_oracle

    rng = np.random.default_rng(0)
    in_dim, hidden, layers, out = 19, 64, 4, 4
    m = S.MLP(in_dim, out, hidden=hidden, layers=layers, max_batch=128, seed=3)
    flat = m.get_params()
    X = rng.standard_normal((96, in_dim)).astype(np.float32)
    T = rng.standard_normal((96, out)).astype(np.float32)
    loss, g = m.loss_and_grads(X, T)
    dims = [in_dim] + [hidden] * layers + [out]
    loss_ref, g_ref, _ = mlp_oracle.loss_and_grads(flat, dims, X, T)
    assert loss == pytest.approx(loss_ref, rel=1e-4)
    # per layer: relative error of the weight and bias gradients
    off = 0
    for din, dout in zip(dims[:-1], dims[1:]):
        for size in (din * dout, dout):
            a, b = g[off:off + size], g_ref[off:off + size]
            assert np.linalg.norm(a - b) <= 1e-3 * np.linalg.norm(b) + 1e-9, (din, dout, size)
            off += size
    assert off == m.n_params


@pytest.mark.gpu
def test_mlp_training_fits_a_smooth_map():
    rng = np.random.default_rng(1)
    X = rng.random((4096, 3)).astype(np.float32)
    Y = np.stack([np.sin(3 * X[:, 0]) + X[:, 1] ** 2, X[:, 2] * X[:, 0] - 0.5 * X[:, 1]], 1).astype(np.float32)
    m = S.MLP(3, 2, hidden=128, layers=3, max_batch=256, seed=0)
    losses = m.fit(X[:3584], Y[:3584], epochs=40, batch=128, lr=2e-3)
    assert losses[-1] < 0.05 * losses[0]
    err = m.predict(X[3584:]) - Y[3584:]
    assert np.sqrt(np.mean(err ** 2)) < 0.05


@pytest.mark.gpu
def test_screening_picks_better_candidates_than_sampling(golden):
    """The gain of the surrogate: among 8x oversampled candidates, the top
    eighth by predicted cost has a lower simulated cost than the same number
    of candidates taken without the surrogate."""
    g = golden["n10_t12s"]
    N, T, TR, ws, step, remove, exc, nvr, seed = [int(v) for v in g["meta"]]
    cfg = B.Config(nodes=N, max_sims=512, time_steps=T, bold_tr=TR, window_size=ws, window_step=step,
                   bold_remove_s=remove, exc_interhem=bool(exc))
    bounds = S.Bounds()
    spec = S.spectral_summary(g["sc"])
    with B.Plan(cfg, g["sc"], g["emp_fc"], g["emp_fcd"]) as plan:
        mlp, info = S.train_surrogate(plan, bounds, spec, n_train=3000, seed=0, epochs=60)
        assert info["holdout_spearman"] > 0.8, info
        rng = np.random.default_rng(7)
        cand = rng.random((3, 512))
        pred = S.cost_of(mlp.predict(S.features(cand, spec)).astype(np.float64))
        top = np.argsort(pred)[:64]
        true_top = S.cost_of(S.simulate(plan, cand[:, top], bounds))
        true_plain = S.cost_of(S.simulate(plan, cand[:, :64], bounds))
    assert true_top.mean() < true_plain.mean() - 0.05, (true_top.mean(), true_plain.mean())
    assert true_top.min() <= true_plain.min() + 1e-9
