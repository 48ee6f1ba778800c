"""FP32 integrator shapes against the FP64 oracle port, through the C ABI, in
oracle-noise mode (the reference's mt19937 stream, bnm.cpp:38-43, fed to
both).

Every kind of shape the autotuner can pick is forced once (BNM_B200_SHAPE):
the register-SC kernel (N <= 128) at N = 67, 68 and 100, where each lane's SC
block is narrower than its 16-byte-aligned S_E stride (18 of 20, 18 of 20 and
26 of 28 columns; N = 67 with a partly filled last warp), and at N = 128 with
full 32-column blocks, with one and two particles per CTA; the shape the
autotuner picks at the smallest and largest cluster sizes (N = 130, 512), at odd N (133, 379: the
column-split kernel with one padding node) and above 512 (600); and for 128 < N <= 512 the
thread-block-cluster kernels, row-split (1, 2, 4 and 8 CTAs per particle, 8
or 16 nodes per warp) and column-split (2 to 7 rows per lane, 8 to 25 column pairs per
warp, one-CTA clusters with a local S_E exchange included, one or two
particles per cluster), with SC in registers only or split between registers
and shared memory.  Two particles per cluster restart together when either
one's FIC check fails; the other's results must still be those of a run
alone, which the per-particle comparison with the oracle checks.  Bar, on every
particle: BOLD within 1e-3 of its range, FC / FCD within 1e-3, cost within 1e-2.  At least 90 % of the
particles must take the oracle's numerical-FIC decisions (wIE equal up to FP32 rounding); any other
particle is compared with the oracle's final pass from its own final wIE.
"""
import concurrent.futures as cf

import numpy as np
import pytest

import bnm_cuda_b200 as B
from bnm_cuda_b200 import synth

pytestmark = pytest.mark.gpu

# N, T ms, TR, remove s, window, step, max trials, particles
SETUPS = {
    "n67": (67, 11000, 500, 2, 6, 2, 3, 3),
    "n68": (68, 12000, 500, 2, 6, 2, 3, 3),
    "n100": (100, 15000, 500, 2, 10, 2, 10, 3),
    "n128": (128, 11000, 500, 2, 6, 2, 3, 2),
    "n130": (130, 11000, 500, 2, 6, 2, 2, 3),
    "n160": (160, 15000, 500, 2, 10, 2, 10, 3),
    "n400": (400, 11000, 500, 2, 6, 2, 2, 2),
    "n512": (512, 10500, 500, 2, 6, 2, 0, 2),
    # odd node counts (one padding node in the column-split kernel) and N > 512
    "n133": (133, 11000, 500, 2, 6, 2, 3, 3),
    "n379": (379, 11000, 500, 2, 6, 2, 2, 2),
    "n600": (600, 10500, 500, 2, 6, 2, 0, 2),
}
# kind,slots,csize,rpw,kr: kind 0 register-SC (slots particles per CTA); kind 1 row-split (rpw nodes per warp, kr chunks in registers); kind 3
# column-split (slots column pairs per warp, rpw rows per lane, kr pairs in registers); kind 4
# column-split with two particles per cluster
SHAPES = {
    "n67": ["0,1,0,0,0", "0,2,0,0,0"],
    "n68": ["0,1,0,0,0", "0,2,0,0,0"],
    "n100": ["0,1,0,0,0", "0,2,0,0,0"],
    "n128": ["0,1,0,0,0", "0,2,0,0,0"],
    "n160": ["1,0,1,8,4", "1,0,2,8,5", "1,0,4,16,4", "1,0,8,8,4",
             "3,10,2,4,10", "3,8,4,2,8", "3,13,2,4,8",
             # one-CTA clusters: S_E exchanged through local shared memory
             "3,10,1,5,10", "3,12,1,6,12", "3,13,1,7,13",
             # two particles per cluster (three particles: one cluster's second half idles)
             "4,10,2,4,10", "4,10,4,2,10"],
    "n400": ["1,0,4,8,4", "1,0,8,8,8", "1,0,8,16,4", "3,25,4,4,8", "3,13,8,2,13", "3,25,8,2,25",
             "4,25,4,4,25", "4,25,4,4,20", "4,13,8,2,13"],
}
# "auto": the shape the autotuner picks (the smallest and largest node counts of the cluster
# kernels, N = 130 and 512)
SHAPES["n130"] = ["auto"]
SHAPES["n512"] = ["auto"]
SHAPES["n133"] = ["auto", "3,10,1,5,10", "4,13,2,4,13"]  # 134 columns: 6 warps of 2 x 13 pairs
SHAPES["n379"] = ["auto", "4,25,4,4,20"]
SHAPES["n600"] = ["auto"]
KINDS = {0: "register", 1: "cluster", 3: "colsplit", 4: "colsplit2"}


@pytest.fixture(scope="module")
def cases(port):
    out = {}
    for name, (N, T, TR, remove, ws, step, trials, n) in SETUPS.items():
        exc = N % 2 == 0  # the hemisphere split (exc_interhem) needs an even node count
        sc = synth.make_sc(N, 0.3 if N < 300 else 0.1, 7)
        G, wEE, wEI = synth.uniform_params(n, N, seed=21, g=(0.5, 2.0))
        cfg = B.Config(nodes=N, max_sims=n, time_steps=T, bold_tr=TR, window_size=ws, window_step=step,
                       bold_remove_s=remove, exc_interhem=exc, max_fic_trials=trials, noise_mode=B.NOISE_HOST)
        s = cfg.sizes()
        noise = port.port_noise(410, s["noise_len"])
        wie0 = np.stack([port.port_analytic_fic(sc, G[i], wEE[i], wEI[i])[0] for i in range(n)])

        def one(i):
            return port.port_integrate(sc, G[i], wEE[i], wEI[i], wie0[i], time_steps=T, bold_tr=TR,
                                       n_vols_remove=s["n_vols_remove"], noise=noise, max_fic_trials=trials)

        with cf.ThreadPoolExecutor(n) as ex:  # the port releases the GIL
            ref = list(ex.map(one, range(n)))
        bold = np.stack([r["bold"] for r in ref])
        kept = bold[:, s["n_vols_remove"]:]
        fc = np.stack([port.port_fc_tril(k, exc) for k in kept])
        fcd = np.stack([port.port_fcd_tril(k, step, ws, exc) for k in kept])
        rng = np.random.default_rng(5)
        emp_fc, emp_fcd = rng.uniform(-0.2, 0.8, fc.shape[1]), rng.uniform(-0.3, 1.0, 500)
        cost = np.array([port.port_gof(k, step, ws, emp_fc, emp_fcd, exc)["cost"] for k in kept])
        out[name] = dict(cfg=cfg, sc=sc, G=G, wEE=wEE, wEI=wEI, wie0=wie0, noise=noise, bold=bold, fc=fc, fcd=fcd,
                         cost=cost, emp_fc=emp_fc, emp_fcd=emp_fcd, trials=np.array([r["trials"] for r in ref]),
                         wIE=np.stack([r["wIE"] for r in ref]))
    return out


def _reference_for_every_particle(r, c, port):
    """The oracle's values for the particles whose numerical FIC took its
    decisions (at least 90 % of them, all in these small batches); the
    oracle's final pass from the device's own final wIE for the others."""
    cfg = c["cfg"]
    s = cfg.sizes()
    ref = dict(bold=c["bold"], fc=c["fc"], fcd=c["fcd"], cost=c["cost"])

    def rerun(i, wie):
        return port.port_final_pass(c["sc"], c["G"][i], c["wEE"][i], c["wEI"][i], wie, time_steps=cfg.time_steps,
                                    bold_tr=cfg.bold_tr, n_vols_remove=s["n_vols_remove"], step=cfg.window_step,
                                    window_size=cfg.window_size, emp_fc=c["emp_fc"], emp_fcd=c["emp_fcd"],
                                    exc=bool(cfg.exc_interhem), noise=c["noise"])

    return port.every_particle_reference(r, ref, c["trials"], c["wIE"], floor=0.9, rerun=rerun)


@pytest.mark.parametrize("name,shape", [(k, s) for k in SHAPES for s in SHAPES[k]])
def test_cluster_shape_matches_fp64_oracle(name, shape, cases, port, monkeypatch):
    c = cases[name]
    if shape == "auto":
        monkeypatch.delenv("BNM_B200_SHAPE", raising=False)
    else:
        monkeypatch.setenv("BNM_B200_SHAPE", shape)
    with B.Plan(c["cfg"], c["sc"], c["emp_fc"], c["emp_fcd"], host_noise=c["noise"]) as p:
        r = p.run(c["G"], c["wEE"], c["wEI"], c["wie0"] if not c["cfg"].do_fic else None)
        info = p.integrator()
    if shape == "auto":
        assert info["kind"] in ("cluster", "colsplit", "colsplit2") and info["tried"] >= 2, info
    else:
        k = [int(v) for v in shape.split(",")]
        assert info["kind"] == KINDS[k[0]], info
        assert (info["slots"], info["csize"], info["rpw"], info["kr"]) == tuple(k[1:]), info
    ref, same = _reference_for_every_particle(r, c, port)
    span = np.ptp(ref["bold"], axis=1, keepdims=True) + 1e-12
    err = (np.abs(r["bold"] - ref["bold"]) / span).max(axis=(1, 2))
    assert err.max() < 1e-3, (err, same)
    np.testing.assert_allclose(r["fc"], ref["fc"], atol=1e-3)
    np.testing.assert_allclose(r["fcd"], ref["fcd"], atol=1e-3)
    np.testing.assert_allclose(r["cost"], ref["cost"], atol=1e-2)


def test_autotuner_picks_a_timed_cluster_shape(cases):
    c = cases["n160"]
    with B.Plan(c["cfg"], c["sc"], c["emp_fc"], c["emp_fcd"], host_noise=c["noise"]) as p:
        r1 = p.run(c["G"], c["wEE"], c["wEI"])
        info = p.integrator()
        r2 = p.run(c["G"], c["wEE"], c["wEI"])  # tuned once per batch size
        assert p.integrator() == info
    assert info["kind"] in ("cluster", "colsplit", "colsplit2") and info["tried"] >= 4, info
    np.testing.assert_array_equal(r1["cost"], r2["cost"])


@pytest.mark.parametrize("N,shape", [(160, "3,10,2,4,10"), (160, "1,0,2,8,5"), (133, "4,13,2,4,13")])
def test_cluster_kernels_draw_the_philox_table_values(N, shape, monkeypatch):
    """The cluster kernels draw their Philox noise by block, one millisecond at a
    time, instead of copying it from a table (their default); with the table
    (BNM_B200_NOISE_SOURCE=table) they stream the same values.  Results must be
    bit-identical, row-split and column-split, odd N (padding node) included."""
    sc = synth.make_sc(N, 0.3, 7)
    G, wEE, wEI = synth.uniform_params(3, N, seed=21, g=(0.5, 2.0))
    cfg = B.Config(nodes=N, max_sims=3, time_steps=11000, bold_tr=500, window_size=6, window_step=2,
                   bold_remove_s=2, exc_interhem=N % 2 == 0, max_fic_trials=2, noise_mode=B.NOISE_PHILOX)
    s = cfg.sizes()
    rng = np.random.default_rng(3)
    emp_fc, emp_fcd = rng.uniform(-0.2, 0.8, s["n_pairs"]), rng.uniform(-0.3, 1.0, 200)
    monkeypatch.setenv("BNM_B200_SHAPE", shape)
    out = []
    for source in ("inline", "table"):
        monkeypatch.setenv("BNM_B200_NOISE_SOURCE", source)
        with B.Plan(cfg, sc, emp_fc, emp_fcd) as p:
            out.append(p.run(G, wEE, wEI))
    for k in ("cost", "bold", "w_ie", "fic_penalty", "ext_means"):
        np.testing.assert_array_equal(out[0][k], out[1][k], err_msg=k)
