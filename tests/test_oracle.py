"""The oracle, pinned before it is trusted (CPU only).

oracle/libbnm_port.so is this project's CPU restatement of the reference's
path.  Here it is checked against the reference's own outputs recorded in
tests/golden (made by tests/golden/make_golden.py from the reference sources
compiled in oracle/_ref): bit for bit on the goodness-of-fit cost and FIC
penalty in both the double and the USE_FLOATS build, on the reference's text
outputs to their printed precision, and on its analysis and analytic-FIC
functions.  The GSL / libks stand-ins are cross-checked against numpy/scipy.
When the reference build is present, a fresh random case is also compared
live.
"""
import numpy as np
import pytest

CASES = ["n10_t12s", "n20_t25s_tr500", "n16_t15s_allpairs", "cfg0_n100_t65s"]


def _meta(g):
    return [int(v) for v in g["meta"]]


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("fp32", [False, True])
def test_port_reproduces_reference_costs_bit_for_bit(case, fp32, golden, port):
    g = golden[case]
    N, T, TR, ws, step, remove, exc, nvr, seed = _meta(g)
    r = port.port_run_batch(g["sc"], g["G"], g["wEE"], g["wEI"], np.zeros_like(g["wEE"]), time_steps=T, bold_tr=TR,
                            n_vols_remove=nvr, seed=seed, window_step=step, window_size=ws, emp_fc=g["emp_fc"],
                            emp_fcd=g["emp_fcd"], exc=bool(exc), fp32=fp32)
    tag = "f32" if fp32 else "f64"
    np.testing.assert_array_equal(r["cost"], g[f"ref_cost_{tag}"])
    np.testing.assert_array_equal(r["fic_penalty"], g[f"ref_pen_{tag}"])
    np.testing.assert_array_equal(r["trials"], g[f"port_trials_{tag}"])


@pytest.mark.parametrize("case", CASES)
def test_port_matches_reference_text_outputs(case, golden, port):
    g = golden[case]
    N, T, TR, ws, step, remove, exc, nvr, seed = _meta(g)
    np.testing.assert_allclose(g["port_bold"], g["ref_bold_txt"], atol=5.1e-8)   # "%.7f"
    np.testing.assert_allclose(g["port_wIE_f64"], g["ref_wIE_txt"], atol=5.1e-7)  # "%f"
    np.testing.assert_array_equal(g["port_trials_f64"], g["ref_ntrials"])
    np.testing.assert_array_equal(g["port_failed_f64"], g["ref_failed"])
    # the extended r_E series (bnm.cpp:212-226) against a fresh port run
    import concurrent.futures as cf

    def one(i):
        return port.port_integrate(g["sc"], g["G"][i], g["wEE"][i], g["wEI"][i], g["ref_wIE_analytic"][i],
                                   time_steps=T, bold_tr=TR, n_vols_remove=nvr, seed=seed)

    with cf.ThreadPoolExecutor(len(g["G"])) as ex:  # the port releases the GIL
        outs = list(ex.map(one, range(len(g["G"]))))
    for i, o in enumerate(outs):
        np.testing.assert_array_equal(o["bold"], g["port_bold"][i])
        np.testing.assert_allclose(o["ext"][2], g["ref_rE_txt"][i][nvr:].mean(0), atol=1e-6)


@pytest.mark.parametrize("case", CASES)
def test_port_analysis_matches_reference_functions(case, golden, port):
    g = golden[case]
    N, T, TR, ws, step, remove, exc, nvr, seed = _meta(g)
    for i in range(len(g["G"])):
        kept = g["port_bold"][i][nvr:]
        np.testing.assert_array_equal(port.port_fc_tril(kept, exc=bool(exc)), g["ref_fc"][i])
        np.testing.assert_array_equal(port.port_fcd_tril(kept, step, ws, exc=bool(exc)), g["ref_fcd"][i])
        gof = port.port_gof(kept, step, ws, g["emp_fc"], g["emp_fcd"], exc=bool(exc))
        assert gof["cost"] == g["ref_gof"][i]


@pytest.mark.parametrize("case", CASES)
def test_port_analytic_fic_matches_reference(case, golden, port):
    g = golden[case]
    for i in range(len(g["G"])):
        w, u = port.port_analytic_fic(g["sc"], g["G"][i], g["wEE"][i], g["wEI"][i])
        assert u == bool(g["ref_unstable"][i])
        if not u:
            np.testing.assert_array_equal(w, g["ref_wIE_analytic"][i])


def test_inline_noise_equals_precomputed_stream(port, golden):
    """bnm.cpp draws noise inline; the GPU reference reads a precomputed array
    (run_CMAES.cpp:640-657).  Both are the same stream, FIC restarts included."""
    g = golden["n10_t12s"]
    N, T, TR, ws, step, remove, exc, nvr, seed = _meta(g)
    nz = port.port_noise(seed, N * (T + 1) * 20)
    for i in range(2):
        a = port.port_integrate(g["sc"], g["G"][i], g["wEE"][i], g["wEI"][i], g["ref_wIE_analytic"][i],
                                time_steps=T, bold_tr=TR, n_vols_remove=nvr, seed=seed)
        b = port.port_integrate(g["sc"], g["G"][i], g["wEE"][i], g["wEI"][i], g["ref_wIE_analytic"][i],
                                time_steps=T, bold_tr=TR, n_vols_remove=nvr, noise=nz)
        np.testing.assert_array_equal(a["bold"], b["bold"])
        assert a["trials"] == b["trials"]


# ------------------------------------------------ GSL / libks stand-ins
def test_ks_matches_scipy(port):
    from scipy.stats import ks_2samp

    rng = np.random.default_rng(0)
    cases = [(rng.normal(size=200), rng.normal(0.2, 1.3, size=350)),
             (rng.integers(0, 5, 100).astype(float), rng.integers(0, 7, 80).astype(float)),  # heavy ties
             (np.array([0.5]), np.array([0.1, 0.5, 0.9])),
             (np.round(rng.uniform(-1, 1, 500), 2), np.round(rng.uniform(-1, 1, 300), 2))]
    for x, y in cases:
        assert port.port_ks(x, y) == pytest.approx(ks_2samp(x, y).statistic, abs=1e-15)


def test_fc_matches_numpy(port):
    rng = np.random.default_rng(1)
    bold = rng.normal(size=(80, 12)) + rng.normal(size=12)
    fc = port.port_fc_tril(bold, exc=False)
    c = np.corrcoef(bold.T)
    i, j = np.tril_indices(12, -1)
    order = np.lexsort((j, i))  # i outer, j inner (check_fit.cpp:37-39)
    np.testing.assert_allclose(fc, c[i[order], j[order]], atol=1e-13)
    fc_exc = port.port_fc_tril(bold, exc=True)
    keep = ~((i[order] < 6) ^ (j[order] < 6))
    np.testing.assert_allclose(fc_exc, c[i[order], j[order]][keep], atol=1e-13)


def test_analytic_fic_root_matches_brentq(port):
    """The Brent solve of fic.cpp:71-100 against scipy's brentq on the same
    equation; the reference stops on a 1e-3 relative bracket."""
    from scipy.optimize import brentq

    a_I, b_I, d_I = 615.0, 177.0, 0.087
    phi = lambda x: (a_I * x - b_I) / (1 - np.exp(-d_I * (a_I * x - b_I)))
    sc = np.zeros((2, 2))
    for wEI in (0.05, 0.2, 0.5, 0.75):
        f = lambda x: 0.382 * 0.7 + wEI * 0.1647572075 - 1.0 * 1.0 * 0.01 * phi(x) - x
        root = brentq(f, 0.0, 2.0, xtol=1e-14)
        w, u = port.port_analytic_fic(sc, 0.0, np.full(2, 0.2), np.full(2, wEI))
        assert not u
        # recover I from wIE: wIE = -(1/S_I) (I_E_ss - I0_E - wEE S_E_ss), S_I = phi(I) * 0.01
        S_I = -(0.3773805650 - 0.382 - 0.2 * 0.1647572075) / w[0]
        assert S_I == pytest.approx(phi(root) * 0.01, rel=2e-3)


# ------------------------------------------------ live reference (optional)
def _live_case():
    from bnm_cuda_b200 import synth
    from oracle import ref

    N, T, TR = 12, 11000, 1000
    sc = synth.make_sc(N, 0.4, 11)
    rng = np.random.default_rng(12)
    G = rng.uniform(0.5, 4, 3)
    wEE = np.repeat(rng.uniform(0.05, 0.75, 3)[:, None], N, 1)
    wEI = np.repeat(rng.uniform(0.05, 0.75, 3)[:, None], N, 1)
    P = N * (N - 1) // 2 - (N // 2) ** 2
    efc, efcd = rng.uniform(-0.2, 0.8, P), rng.uniform(-0.5, 1, 15)
    kw = dict(time_steps=T, bold_tr=TR, emp_fc=efc, emp_fcd=efcd, window_step=1, window_size=3)
    c, p = ref.ref_run_simulations(sc, G, wEE, wEI, np.zeros_like(wEE), rand_seed=5, max_fic_trials=10, **kw)
    r = ref.port_run_batch(sc, G, wEE, wEI, np.zeros_like(wEE), n_vols_remove=2, seed=5, **kw)
    return c, p, r["cost"], r["fic_penalty"]


def test_live_reference_vs_port():
    from oracle import ref

    if not ref.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    c, p, c2, p2 = ref.run_isolated(_live_case, env={"BNM_BOLD_REMOVE": 2})
    np.testing.assert_array_equal(c, c2)
    np.testing.assert_array_equal(p, p2)


@pytest.mark.parametrize("het", [(), ("wee",), ("wei",), ("wee", "wei"), ("wee", "wie", "wei")])
def test_calculate_params_matches_reference_bit_for_bit(het):
    """The library's parameter expansion (bnm_calculate_params, used by the
    run_CMAES_gpu driver) against the reference's own calculate_params
    (run_CMAES.cpp:61-143, compiled unmodified in oracle/_ref): base values,
    per-node map scaling base * (1 + sum_m coef_m map_m[j]) and the shift of
    a regional parameter whose smallest node value falls below 0.001.  Maps
    of both kinds the driver accepts (min-max normalised to [0, 1] and
    z-scored), coefficients drawn across the driver's scale bounds, so both
    shifted and unshifted expansions occur."""
    from oracle import ref

    if not ref.ref_available():
        pytest.skip("reference build missing (make -C oracle)")
    import bnm_cuda_b200 as B

    rng = np.random.default_rng(11)
    N = 100
    shifted = 0
    for trial in range(40):
        n_maps = 1 + trial % 3
        maps = []
        for m in range(n_maps):
            x = rng.standard_normal(N)
            maps.append((x - x.min()) / (x.max() - x.min()) if m % 2 == 0 else (x - x.mean()) / x.std())
        maps = np.array(maps)
        # coefficient ranges as run_CMAES.cpp:272-289 derives them (min-max maps: [0, scale_max_minmax];
        # z-scored: [ceil(-1/max, 0.01), floor(-1/min, 0.01)]), stretched a little past them
        zs = np.arange(n_maps) % 2 == 1
        lo, hi = np.full(n_maps, -0.5), np.full(n_maps, 5.0)
        lo[zs] = np.ceil(-1 / maps[zs].max(1) / 0.01) * 0.01 - 0.2
        hi[zs] = np.floor(-1 / maps[zs].min(1) / 0.01) * 0.01 + 0.2
        scales = rng.uniform(lo, hi, (3, n_maps))
        G, wee, wie, wei = rng.uniform(0.5, 4), rng.uniform(0.001, 0.75), rng.uniform(0, 2), rng.uniform(0.001, 0.75)
        mask = sum(1 << B.LOCAL_PARAMS.index(h) for h in het)
        want = ref.ref_calculate_params(N, mask, maps, G, wee, wie, wei, scales)
        got = B.calculate_params(N, G, wee, wie, wei, het=het, maps=maps, scales=scales)
        assert got[0] == want[0]
        for a, b in zip(got[1:], want[1:]):
            np.testing.assert_array_equal(a, b)
        for h in het:
            k = {"wee": 1, "wei": 2, "wie": 3}[h]
            shifted += int(np.isclose(want[k].min(), 0.001))
    if het:
        assert shifted > 0  # the 0.001 shift was exercised
