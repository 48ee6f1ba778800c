"""Regenerates the golden fixtures in this directory from the reference itself.

    python tests/golden/make_golden.py [case ...] # simulation fixtures (all, or the named ones)
    python tests/golden/make_golden.py --cmaes    # CMA-ES fixtures

Needs the reference build in oracle/_ref (``make -C oracle``, which compiles
the reference's unmodified CPU sources against oracle/compat) and the port
(oracle/libbnm_port.so).  For each case it records:

* inputs: SC, per-particle G / wEE / wEI, empirical FC / FCD targets (made by
  the port at G=2.0, wEE=0.3, wEI=0.2 with noise seed 1, the same-model
  targets of the single-simulation workload);
* the reference's run_simulations (bnm.cpp:431-466) goodness-of-fit cost and
  FIC penalty, in its double build and in its USE_FLOATS build;
* the reference's per-particle text outputs (bnm.cpp:292-388: BOLD, wIE,
  FIC trial count / failure flag, extended r_E series) with save_output on;
* the reference's analytical_fic (fic.cpp:130-207) and fc_tril / fcd_tril /
  check_fit_bold (check_fit.cpp) on the port's BOLD, after checking that the
  port reproduces the reference's cost bit for bit.

The reference reads BNM_* at load time, so each case runs in a fresh process.
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
sys.path.insert(0, ROOT)

CASES = {
    # name: (N, T, TR, ws, step, bold_remove_s, exc, n_particles, density, seed)
    "n10_t12s": dict(N=10, T=12000, TR=1000, ws=4, step=1, remove=2, exc=1, n=6, density=0.5, seed=3),
    "n20_t25s_tr500": dict(N=20, T=25000, TR=500, ws=6, step=2, remove=2, exc=1, n=6, density=0.3, seed=4),
    "n16_t15s_allpairs": dict(N=16, T=15000, TR=1000, ws=3, step=1, remove=1, exc=0, n=4, density=0.4, seed=5),
    # the single-simulation workload at full size: N = 100 (30 % density SC, seed 0), 65 s at TR 1 s
    # (66 frames, 5 s removed), window 10 step 2 (26 windows, 325 FCD entries); particle 0 is its
    # G = 1.5, wEE = 0.21, wEI = 0.15
    "cfg0_n100_t65s": dict(N=100, T=65000, TR=1000, ws=10, step=2, remove=5, exc=1, n=4, density=0.3, seed=0),
}


def _case(name, c):
    from oracle import ref
    from bnm_cuda_b200 import synth

    N, T, TR = c["N"], c["T"], c["TR"]
    nvr = c["remove"] * 1000 // TR
    sc = synth.make_sc(N, c["density"], c["seed"])
    rng = np.random.default_rng(100 + c["seed"])
    n = c["n"]
    G = rng.uniform(0.5, 4.0, n)
    G[0] = 1.5
    we = rng.uniform(0.05, 0.75, n)
    wi = rng.uniform(0.05, 0.75, n)
    we[0], wi[0] = 0.21, 0.15
    wEE, wEI = np.repeat(we[:, None], N, 1), np.repeat(wi[:, None], N, 1)
    wIE0 = np.zeros((n, N))
    # same-model targets (port, double, noise seed 1)
    w_t, uns = ref.port_analytic_fic(sc, 2.0, np.full(N, 0.3), np.full(N, 0.2))
    if uns:
        w_t = np.ones(N)
    tgt = ref.port_integrate(sc, 2.0, np.full(N, 0.3), np.full(N, 0.2), w_t, time_steps=T, bold_tr=TR,
                             n_vols_remove=nvr, seed=1)
    kept = tgt["bold"][nvr:]
    emp_fc = ref.port_fc_tril(kept, exc=bool(c["exc"]))
    emp_fcd = ref.port_fcd_tril(kept, c["step"], c["ws"], exc=bool(c["exc"]))

    out = dict(sc=sc, G=G, wEE=wEE, wEI=wEI, emp_fc=emp_fc, emp_fcd=emp_fcd,
               meta=np.array([N, T, TR, c["ws"], c["step"], c["remove"], c["exc"], nvr, 410]))
    kw = dict(time_steps=T, bold_tr=TR, rand_seed=410, max_fic_trials=10, emp_fc=emp_fc, emp_fcd=emp_fcd,
              window_step=c["step"], window_size=c["ws"])
    for fp32 in (False, True):
        tag = "f32" if fp32 else "f64"
        cost, pen = ref.ref_run_simulations(sc, G, wEE, wEI, wIE0, fp32=fp32, **kw)
        out[f"ref_cost_{tag}"], out[f"ref_pen_{tag}"] = cost, pen
        # port must reproduce it bit for bit
        pr = ref.port_run_batch(sc, G, wEE, wEI, wIE0, time_steps=T, bold_tr=TR, n_vols_remove=nvr, seed=410,
                                window_step=c["step"], window_size=c["ws"], emp_fc=emp_fc, emp_fcd=emp_fcd,
                                exc=bool(c["exc"]), fp32=fp32)
        assert np.array_equal(pr["cost"], cost), (name, tag, pr["cost"], cost)
        assert np.array_equal(pr["fic_penalty"], pen), (name, tag)
        out[f"port_wIE_{tag}"], out[f"port_trials_{tag}"] = pr["wIE"], pr["trials"]
        out[f"port_failed_{tag}"] = pr["failed"]
    # per-particle reference text outputs (double build)
    with tempfile.TemporaryDirectory() as d:
        bold_txt, wie_txt, ntr, fl, rE_txt = [], [], [], [], []
        for i in range(n):
            pre = os.path.join(d, f"p{i}")
            ref.ref_run_simulations(sc, G[i:i + 1], wEE[i:i + 1], wEI[i:i + 1], wIE0[i:i + 1], out_prefix=pre,
                                    save_output=True, **kw)
            bold_txt.append(np.loadtxt(pre + "_bold.txt"))
            wie_txt.append(np.loadtxt(pre + "_w_IE.txt"))
            ntr.append(int(open(pre + "_fic_ntrials.txt").read().split()[0]))
            fl.append(int(open(pre + "_fic_failed.txt").read()))
            rE_txt.append(np.loadtxt(pre + "_r_E.txt"))
        out["ref_bold_txt"], out["ref_wIE_txt"] = np.array(bold_txt), np.array(wie_txt)
        out["ref_ntrials"], out["ref_failed"], out["ref_rE_txt"] = np.array(ntr), np.array(fl), np.array(rE_txt)
    # reference analysis functions on the (bit-identical) port BOLD of each particle
    fcs, fcds, costs, bolds, wfic, unst = [], [], [], [], [], []
    for i in range(n):
        w0, u = ref.ref_analytical_fic(sc, G[i], wEE[i], wEI[i])
        wp, up = ref.port_analytic_fic(sc, G[i], wEE[i], wEI[i])
        assert u == up and (u or np.array_equal(w0, wp)), (name, i)
        wfic.append(w0 if not u else np.ones(N))
        unst.append(u)
        r = ref.port_integrate(sc, G[i], wEE[i], wEI[i], wfic[-1], time_steps=T, bold_tr=TR, n_vols_remove=nvr,
                               seed=410)
        bolds.append(r["bold"])
        k = r["bold"][nvr:]
        fcs.append(ref.ref_fc_tril(k, exc=bool(c["exc"])))
        fcds.append(ref.ref_fcd_tril(k, c["step"], c["ws"], exc=bool(c["exc"])))
        costs.append(ref.ref_check_fit_bold(k, c["step"], c["ws"], emp_fc, emp_fcd, exc=bool(c["exc"])))
    out["ref_wIE_analytic"], out["ref_unstable"] = np.array(wfic), np.array(unst)
    out["ref_fc"], out["ref_fcd"], out["ref_gof"] = np.array(fcs), np.array(fcds), np.array(costs)
    assert np.array_equal(np.array(costs), out["ref_cost_f64"]), (name, costs, out["ref_cost_f64"])
    out["port_bold"] = np.array(bolds)
    np.savez_compressed(os.path.join(ROOT, "tests", "golden", f"{name}.npz"), **out)
    return name


def _env(c):
    return {"BNM_BOLD_REMOVE": c["remove"], "BNM_EXC_INTERHEM": c["exc"]}


if __name__ == "__main__" and "--cmaes" not in sys.argv:
    from oracle import ref

    only = [a for a in sys.argv[1:] if a in CASES]
    for name, c in CASES.items():
        if not only or name in only:
            print(ref.run_isolated(_case, name, c, env=_env(c)))


def cmaes_objective(X):
    """Deterministic test objective on [0,1]^D (columns are particles)."""
    D = X.shape[0]
    t = np.linspace(0.2, 0.8, D)[:, None]
    return ((X - t) ** 2).sum(0) + 0.05 * np.sin(7 * X).sum(0)


def _cmaes_case(lam, dim, seed, it_max, variante):
    """The reference's CMAES_Points (cmaes.cpp) driven as run_CMAES.cpp main()
    does, on cmaes_objective: every generation's feasible samples, penalised
    costs and the final best point."""
    from oracle import ref

    r = ref.ref_lib()
    r.ref_cmaes_setup(lam, dim, seed, it_max)
    feas_all, pen_all = [], []
    while r.ref_cmaes_it() < it_max:
        fe = np.zeros(dim * lam)
        r.ref_cmaes_get(fe, np.zeros(dim * lam), np.zeros(dim * lam))
        fe = fe.reshape(dim, lam)
        pen = np.zeros(lam)
        r.ref_cmaes_tell(cmaes_objective(fe), pen)
        feas_all.append(fe)
        pen_all.append(pen)
    best = np.zeros(dim + 1)
    r.ref_cmaes_best(best)
    return dict(feas=np.array(feas_all), penalized=np.array(pen_all), best=best,
                meta=np.array([lam, dim, seed, it_max, variante]))


def make_cmaes_golden():
    from oracle import ref

    for lam, dim, seed, it_max, var in [(10, 3, 1, 40, 6), (16, 9, 7, 25, 16)]:
        out = ref.run_isolated(_cmaes_case, lam, dim, seed, it_max, var, env={"BNM_CMAES_VARIANTE": var})
        np.savez_compressed(os.path.join(ROOT, "tests", "golden", f"cmaes_l{lam}_d{dim}_v{var}.npz"), **out)
        print("cmaes", lam, dim, var, len(out["feas"]))


if __name__ == "__main__" and "--cmaes" in sys.argv:
    make_cmaes_golden()
