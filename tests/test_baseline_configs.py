"""Parity at the benchmark's own sizes (the one-generation CMA-ES workload:
N = 100, 450 s of model time, TR 0.72 s, 30 s removed, window 44 step 1,
541 windows, 2450 pairs, 146,070 FCD entries, FIC on), through the C ABI.

1. Stage-wise: the FP32 product path integrates a batch; its own BOLD is then
   analysed by the FP64 oracle (check_fit.cpp:19-217 restated in
   oracle/bnm_port.cpp).  FC, every FCD entry, the KS distance and the cost
   must agree within 1e-3 for each Gram arithmetic (split BF16 on tensor
   cores, the default; FP32 SIMT).  The same BOLD in, so the difference is the
   device analysis alone.
2. Full horizon: FP32 integration against the FP64 reference-order kernel
   (pinned to the reference's double build at 1e-9 on the golden fixtures) on
   the same noise over the whole 450 s, on 16 particles.  A particle whose FIC
   took different decisions in the two arithmetics is compared with an FP64
   run from the FP32 run's final wIE (numerical FIC off), so every particle is
   compared.  The two trajectories are not expected to stay step for step
   equal over 4.5 M noisy substeps; the bounds below are on the statistics the
   fit uses (stated with the test).

Inputs are the benchmark's: SC seed 0 (30 % density), particles from seed 1
on G [0.5, 4], wEE / wEI [0.05, 0.75], Philox noise seed 410, targets the
model's own FC / FCD at G = 2, wEE = 0.3, wEI = 0.2 (noise seed 1).
"""
import concurrent.futures as cf

import numpy as np
import pytest

import bnm_cuda_b200 as B
from bnm_cuda_b200 import synth

pytestmark = pytest.mark.gpu

N, T, TR, WS, STEP, REMOVE = 100, 450_000, 720, 44, 1, 30


def _cfg(n, **kw):
    return B.Config(nodes=N, max_sims=n, time_steps=T, bold_tr=TR, window_size=WS, window_step=STEP,
                    bold_remove_s=REMOVE, noise_seed=410, **kw)


@pytest.fixture(scope="module")
def workload():
    sc = synth.make_sc(N, 0.3, 0)
    G, wEE, wEI = synth.uniform_params(256, N, 1)
    cfg = B.Config(**{**_cfg(1).__dict__, "noise_seed": 1})
    s = cfg.sizes()
    assert (s["frames"], s["n_vols_remove"], s["n_windows"], s["n_pairs"], s["n_fcd"]) == (626, 41, 541, 2450, 146070)
    with B.Plan(cfg, sc, np.zeros(s["n_pairs"]), np.zeros(s["n_fcd"])) as p:
        t = p.run(2.0, 0.3, 0.2, outputs=("fc", "fcd"))
    return dict(sc=sc, G=G, wEE=wEE, wEI=wEI, emp_fc=t["fc"][0], emp_fcd=t["fcd"][0], nvr=s["n_vols_remove"])


@pytest.mark.parametrize("gram", [B.GRAM_AUTO, B.GRAM_F32])
def test_config1_analysis_stagewise_within_1e3_of_fp64_oracle(workload, port, gram):
    w = workload
    n = 4
    with B.Plan(_cfg(n, gram=gram), w["sc"], w["emp_fc"], w["emp_fcd"]) as p:
        r = p.run(w["G"][:n], w["wEE"][:n], w["wEI"][:n], outputs=("bold", "fc", "fcd"))
    assert r["fcd"].shape == (n, 146070)

    def oracle(i):
        kept = r["bold"][i, w["nvr"]:]
        fit = port.port_gof(kept, STEP, WS, w["emp_fc"], w["emp_fcd"])
        return port.port_fc_tril(kept), port.port_fcd_tril(kept, STEP, WS), fit

    with cf.ThreadPoolExecutor(n) as ex:  # the port releases the GIL
        ref = list(ex.map(oracle, range(n)))
    for i, (fc, fcd, fit) in enumerate(ref):
        assert np.abs(r["fc"][i] - fc).max() < 1e-3
        assert np.abs(r["fcd"][i] - fcd).max() < 1e-3
        assert abs(r["fcd_ks"][i] - fit["fcd_ks"]) < 1e-3
        assert abs(r["fc_corr"][i] - fit["fc_corr"]) < 1e-3
        assert abs(r["cost"][i] - fit["cost"]) < 1e-3


def full_horizon_statistics(workload, n=16):
    """FP32 product path vs FP64 reference-order kernel over the full 450 s
    on the first n particles, same Philox noise.  Returns per-particle |d cost|,
    |d KS|, |d FC correlation|, the Pearson correlation between the two FC
    vectors, the max |d FC| entry, and which particles needed the FP64 rerun
    from the FP32 run's final wIE."""
    w = workload
    out = ("w_ie", "fc", "fcd")
    with B.Plan(_cfg(n), w["sc"], w["emp_fc"], w["emp_fcd"]) as p:
        r32 = p.run(w["G"][:n], w["wEE"][:n], w["wEI"][:n], outputs=out)
    with B.Plan(_cfg(n, precision=B.PREC_F64), w["sc"], w["emp_fc"], w["emp_fcd"]) as p:
        r64 = p.run(w["G"][:n], w["wEE"][:n], w["wEI"][:n], outputs=out)
    same = (r32["fic_ntrials"] == r64["fic_ntrials"]) & (np.abs(r32["w_ie"] - r64["w_ie"]).max(1) < 1e-4)
    if not same.all():
        k = np.flatnonzero(~same)
        with B.Plan(_cfg(len(k), precision=B.PREC_F64, do_fic=False, calculate_fic_penalty=False), w["sc"],
                    w["emp_fc"], w["emp_fcd"]) as p:
            rr = p.run(w["G"][k], w["wEE"][k], w["wEI"][k], r32["w_ie"][k], outputs=out)
        for key in ("cost", "fcd_ks", "fc_corr", "fc", "fcd"):
            r64[key][k] = rr[key]
    fc_r = np.array([np.corrcoef(r32["fc"][i], r64["fc"][i])[0, 1] for i in range(n)])
    return dict(d_cost=np.abs(r32["cost"] - r64["cost"]), d_ks=np.abs(r32["fcd_ks"] - r64["fcd_ks"]),
                d_fc_corr=np.abs(r32["fc_corr"] - r64["fc_corr"]), fc_r=fc_r,
                d_fc_max=np.abs(r32["fc"] - r64["fc"]).max(1), rerun=~same)


def test_config1_full_horizon_fp32_statistics_against_fp64(workload):
    """FP32 product path vs the FP64 reference-order kernel over the whole
    450 s, 16 particles, same noise.  Bounds (about ten times the values
    measured on a B200: max |d cost| 9.3e-6, median 3.3e-7; max |d KS|
    6.8e-6; max |d FC| entry 5.5e-6; FC correlation between the two runs
    >= 1 - 1.3e-10; one particle of 16 took other FIC decisions and was
    compared through the FP64 rerun from its FP32 wIE)."""
    s = full_horizon_statistics(workload, n=16)
    assert s["d_cost"].max() < 1e-4 and np.median(s["d_cost"]) < 1e-5, s["d_cost"]
    assert s["d_ks"].max() < 1e-4, s["d_ks"]
    assert s["d_fc_corr"].max() < 1e-5, s["d_fc_corr"]
    assert s["d_fc_max"].max() < 5e-5, s["d_fc_max"]
    assert s["fc_r"].min() > 1 - 1e-8, s["fc_r"]
    assert s["rerun"].sum() <= 3, s["rerun"]  # FIC decisions agree for nearly every particle

