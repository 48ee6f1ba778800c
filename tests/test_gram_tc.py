"""Tensor-core (tcgen05) FC and FCD Grams in BF16 and split BF16 against the
FP64 oracle, through the C ABI.

The three Gram arithmetics run on the same device BOLD (the integrator does
not depend on the Gram setting, so BOLD must be bit-identical), and each FC /
FCD entry is compared with the oracle port's FP64 FC and FCD of that BOLD
(check_fit.cpp:19-134).  Tolerances, absolute on correlations in [-1, 1]:

  F32         FC 1e-6 (FP64 co-moments), FCD 2e-5 (FP32 SIMT Gram)
  BF16        FC 2e-3, FCD 1e-3 (one BF16 rounding per operand value; FC
              series dominated by a few frames, e.g. the BOLD onset when no
              frames are removed, do not average the rounding out, so BF16 FC
              can exceed 1e-3 and split BF16 is the default)
  BF16_SPLIT  FC 1e-5, FCD 1e-5 (hi + lo parts; partial sums of 128 K
              drained from the tensor-core accumulator into FP32)

The KS distance fused into the Gram epilogue must equal the oracle's
two-sample KS of the device's own FCD values (to the last bits of the final
division), and lie within 1e-2
(BF16) / 2e-3 (F32, split) of the KS of the FP64 FCD.
"""
import concurrent.futures as cf

import numpy as np
import pytest

import bnm_cuda_b200 as B
from bnm_cuda_b200 import synth

pytestmark = pytest.mark.gpu

# N, T (ms), TR (ms), window size, step, removed s, exc_interhem
CASES = {
    # 263 windows: 3 row blocks with a ragged last one; 2450 pairs: 39 K tiles (the ring wraps)
    "n100_w263": (100, 250000, 720, 44, 1, 30, True),
    # 160 nodes: 2 FC row blocks, 181 frames: 3 K tiles; 12720 pairs, 54 windows: one diagonal FCD tile
    "n160_allpairs": (160, 100000, 500, 20, 3, 10, False),
}
TOL = {B.GRAM_F32: (1e-6, 2e-5, 2e-3), B.GRAM_BF16: (2e-3, 1e-3, 1e-2), B.GRAM_BF16_SPLIT: (1e-5, 1e-5, 2e-3)}
NAMES = {B.GRAM_F32: "f32", B.GRAM_BF16: "bf16", B.GRAM_BF16_SPLIT: "bf16x3"}


# The precision-stress shape (N = 400, all 79,800 pairs, TR 0.5 s, window 44
# step 1) on 200 s of model time with 10 s removed: 381 frames, 337 windows,
# 56,616 FCD entries, 3 FCD row blocks, 1247 K tiles (cluster integrator).
CONFIG2_SHAPE = (400, 200000, 500, 44, 1, 10, False)


def _run_all(case, n=3):
    N, T, TR, ws, step, remove, exc = CASES[case] if isinstance(case, str) else case
    sc = synth.make_sc(N, 0.3, 5)
    G, wEE, wEI = synth.uniform_params(n, N, seed=11)
    rng = np.random.default_rng(3)
    emp_fc = rng.uniform(-0.2, 0.8, synth.n_pairs(N, exc))
    emp_fcd = rng.uniform(-0.3, 1.0, 4001)
    res = {}
    for gram in TOL:
        cfg = B.Config(nodes=N, max_sims=n, time_steps=T, bold_tr=TR, window_size=ws, window_step=step,
                       bold_remove_s=remove, exc_interhem=exc, gram=gram)
        with B.Plan(cfg, sc, emp_fc, emp_fcd) as p:
            res[gram] = p.run(G, wEE, wEI, outputs=("bold", "fc", "fcd"))
    return cfg, emp_fcd, res


def _grams_against_oracle(case, port, n=3):
    cfg, emp_fcd, res = _run_all(case, n)
    N, T, TR, ws, step, remove, exc = CASES[case] if isinstance(case, str) else case
    nvr = cfg.sizes()["n_vols_remove"]
    bold = res[B.GRAM_F32]["bold"]
    errs = {}
    for gram, r in res.items():
        np.testing.assert_array_equal(r["bold"], bold)

    def oracle(i):
        kept = bold[i][nvr:]
        return port.port_fc_tril(kept, exc=exc), port.port_fcd_tril(kept, step, ws, exc=exc)

    with cf.ThreadPoolExecutor(len(bold)) as ex:  # the port releases the GIL
        ref = list(ex.map(oracle, range(len(bold))))
    for i, (fc64, fcd64) in enumerate(ref):
        ks64 = port.port_ks(emp_fcd, fcd64)
        for gram, r in res.items():
            e = (np.abs(r["fc"][i] - fc64).max(), np.abs(r["fcd"][i] - fcd64).max(), abs(r["fcd_ks"][i] - ks64))
            errs[NAMES[gram]] = np.maximum(errs.get(NAMES[gram], 0), e)
            assert r["fcd_ks"][i] == pytest.approx(port.port_ks(emp_fcd, r["fcd"][i]), abs=1e-12), (NAMES[gram], i)
    print(case, {k: [f"{x:.2e}" for x in v] for k, v in errs.items()})
    for gram in res:
        assert np.all(errs[NAMES[gram]] <= np.array(TOL[gram])), (NAMES[gram], errs[NAMES[gram]])
    return cfg


@pytest.mark.parametrize("case", list(CASES))
def test_tensor_core_grams_against_fp64_oracle(case, port):
    _grams_against_oracle(case, port)


def test_config2_shape_grams_against_fp64_oracle(port):
    """Every Gram arithmetic at the precision-stress workload's node count,
    pair count, TR and window (CONFIG2_SHAPE) against the FP64 oracle
    (check_fit.cpp:19-134 restated) on the same BOLD, two particles."""
    cfg = _grams_against_oracle(CONFIG2_SHAPE, port, n=2)
    s = cfg.sizes()
    assert (s["n_pairs"], s["frames"] - s["n_vols_remove"], s["n_windows"]) == (79800, 381, 337)


def test_staged_chunks_give_the_same_result(monkeypatch):
    """FCD operands staged a few simulations at a time (BNM_B200_GRAM_CHUNK)
    give bit-identical FCD and KS."""
    N, T, TR, ws, step, remove, exc = CASES["n100_w263"]
    sc = synth.make_sc(N, 0.3, 5)
    n = 5
    G, wEE, wEI = synth.uniform_params(n, N, seed=12)
    rng = np.random.default_rng(4)
    emp_fc = rng.uniform(-0.2, 0.8, synth.n_pairs(N, exc))
    emp_fcd = rng.uniform(-0.3, 1.0, 2000)
    cfg = B.Config(nodes=N, max_sims=n, time_steps=T, bold_tr=TR, window_size=ws, window_step=step,
                   bold_remove_s=remove, exc_interhem=exc, gram=B.GRAM_BF16_SPLIT)
    out = []
    for chunk in (None, "2"):
        if chunk:
            monkeypatch.setenv("BNM_B200_GRAM_CHUNK", chunk)
        with B.Plan(cfg, sc, emp_fc, emp_fcd) as p:
            out.append(p.run(G, wEE, wEI, outputs=("fcd",)))
    np.testing.assert_array_equal(out[0]["fcd"], out[1]["fcd"])
    np.testing.assert_array_equal(out[0]["fcd_ks"], out[1]["fcd_ks"])
    np.testing.assert_array_equal(out[0]["cost"], out[1]["cost"])


def test_check_fit_bold_reproduces_the_batch_and_the_oracle(port):
    """bnm_check_fit_bold on the BOLD a batch produced gives that batch's FC,
    FCD, KS and cost (the FIC penalty is a separate output, zero here), and
    agrees with the oracle's check_fit_bold (check_fit.cpp:138-217) on the
    same BOLD."""
    N, T, TR, ws, step, remove, exc = CASES["n100_w263"]
    sc = synth.make_sc(N, 0.3, 5)
    n = 3
    G, wEE, wEI = synth.uniform_params(n, N, seed=13)
    rng = np.random.default_rng(6)
    emp_fc = rng.uniform(-0.2, 0.8, synth.n_pairs(N, exc))
    emp_fcd = rng.uniform(-0.3, 1.0, 3000)
    for gram in TOL:
        cfg = B.Config(nodes=N, max_sims=n, time_steps=T, bold_tr=TR, window_size=ws, window_step=step,
                       bold_remove_s=remove, exc_interhem=exc, gram=gram)
        nvr = cfg.sizes()["n_vols_remove"]
        with B.Plan(cfg, sc, emp_fc, emp_fcd) as p:
            r = p.run(G, wEE, wEI, outputs=("bold", "fc", "fcd"))
            f = p.check_fit_bold(r["bold"][:, nvr:])
        np.testing.assert_array_equal(f["fc"], r["fc"])
        np.testing.assert_array_equal(f["fcd"], r["fcd"])
        np.testing.assert_array_equal(f["fcd_ks"], r["fcd_ks"])
        np.testing.assert_allclose(f["cost"], r["cost"], atol=1e-12)  # the penalty is reported apart
        assert (f["fic_penalty"] == 0).all()
        for i in range(n):
            ref = port.port_gof(r["bold"][i][nvr:], step, ws, emp_fc, emp_fcd, exc=exc)
            assert f["cost"][i] == pytest.approx(ref["cost"], abs=TOL[gram][2] + 1e-3)


@pytest.mark.parametrize("case", list(CASES))
def test_hemisphere_fcd_against_fp64_oracle(case, port):
    """fcd_left / fcd_right (the reference's save_hemis outputs, bnm.cu:436-551):
    FCD over the first and the last (N/2)(N/2-1)/2 pairs of the window-FC
    vectors, each centred over its own pairs, against FP64 from the oracle's
    window FC (FP32 Gram: 1e-4).  Asking for them leaves the batch's FCD and
    cost unchanged, and bnm_check_fit_bold returns the same values."""
    N, T, TR, ws, step, remove, exc = CASES[case]
    sc = synth.make_sc(N, 0.3, 5)
    n = 2
    G, wEE, wEI = synth.uniform_params(n, N, seed=14)
    rng = np.random.default_rng(8)
    emp_fc = rng.uniform(-0.2, 0.8, synth.n_pairs(N, exc))
    emp_fcd = rng.uniform(-0.3, 1.0, 1000)
    cfg = B.Config(nodes=N, max_sims=n, time_steps=T, bold_tr=TR, window_size=ws, window_step=step,
                   bold_remove_s=remove, exc_interhem=exc)
    nvr = cfg.sizes()["n_vols_remove"]
    with B.Plan(cfg, sc, emp_fc, emp_fcd) as p:
        plain = p.run(G, wEE, wEI, outputs=("fcd",))
        r = p.run(G, wEE, wEI, outputs=("bold", "fcd", "fcd_left", "fcd_right"))
        f = p.check_fit_bold(r["bold"][:, nvr:], outputs=("fcd_left", "fcd_right"))
    np.testing.assert_array_equal(r["fcd"], plain["fcd"])
    np.testing.assert_array_equal(r["cost"], plain["cost"])
    np.testing.assert_array_equal(f["fcd_left"], r["fcd_left"])
    np.testing.assert_array_equal(f["fcd_right"], r["fcd_right"])
    h = N // 2
    nh = h * (h - 1) // 2
    for i in range(n):
        kept = r["bold"][i][nvr:]
        _, wfc = port.port_fcd_tril(kept, step, ws, exc=exc, window_fc=True)
        P = wfc.shape[1]
        for sub, got in ((wfc[:, :nh], r["fcd_left"][i]), (wfc[:, P - nh:], r["fcd_right"][i])):
            z = sub - sub.mean(1, keepdims=True)
            z /= np.sqrt((z * z).sum(1, keepdims=True))
            a, b = np.tril_indices(len(z), -1)
            assert np.abs(got - (z @ z.T)[a, b]).max() <= 1e-4
        if exc:  # then the two ranges are exactly the within-hemisphere pairs
            left = port.port_fcd_tril(kept[:, :h], step, ws, exc=False)
            right = port.port_fcd_tril(kept[:, h:], step, ws, exc=False)
            assert np.abs(r["fcd_left"][i] - left).max() <= 1e-4
            assert np.abs(r["fcd_right"][i] - right).max() <= 1e-4


def test_window_tile_tuner_gives_the_same_window_fc(monkeypatch):
    """The window-FC tile (pairs per CTA) is tuned on the first run of a batch
    size; every tile computes the same window FC (each pair's co-moments are
    formed by one thread whatever the tile), so the tuned plan and plans forced
    to the default tile must agree on FC and FCD."""
    N = 40
    sc = synth.make_sc(N, 0.3, 2)
    cfg = B.Config(nodes=N, max_sims=4, time_steps=30000, bold_tr=500, window_size=10, window_step=2,
                   bold_remove_s=2, gram=B.GRAM_F32)
    s = cfg.sizes()
    rng = np.random.default_rng(4)
    emp_fc, emp_fcd = rng.uniform(-0.2, 0.8, s["n_pairs"]), rng.uniform(-0.3, 1.0, 300)
    G, wEE, wEI = synth.uniform_params(4, N, 8)
    with B.Plan(cfg, sc, emp_fc, emp_fcd) as p:
        a = p.run(G, wEE, wEI)
        tile = p.window_tile()
    assert tile["tried"] == 4 and tile["pairs_per_thread"] in (1, 2, 4, 8), tile
    monkeypatch.setenv("BNM_B200_TUNE", "0")
    with B.Plan(cfg, sc, emp_fc, emp_fcd) as p:
        b = p.run(G, wEE, wEI)
        assert p.window_tile()["pairs_per_thread"] == 4
    np.testing.assert_array_equal(a["fc"], b["fc"])
    np.testing.assert_allclose(a["fcd"], b["fcd"], rtol=0, atol=1e-6)
