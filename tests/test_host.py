"""Host-side checks of the C ABI library (no GPU work): it loads, exports every
entry point include/bnm_b200.h declares, derives the reference's sizes, reads
BNM_* like the reference, rejects bad configurations with status codes, and
its CMA-ES reproduces the reference's CMAES_Points bit for bit."""
import os
import re
import subprocess
import sys

import numpy as np
import pytest

import bnm_cuda_b200 as B
from bnm_cuda_b200 import synth

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def test_library_exports_every_declared_symbol():
    hdr = open(os.path.join(ROOT, "include", "bnm_b200.h")).read()
    names = set(re.findall(r"^\s*(?:int|void|int32_t|const char \*)\s*\*?(bnm_\w+)\s*\(", hdr, re.M))
    assert len(names) >= 20
    lib = B.lib()
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", B.LIB_PATH], capture_output=True, text=True).stdout
    for n in names:
        assert re.search(rf"\bT {n}\b", out), n


@pytest.mark.parametrize("w", [synth.CONFIG0, synth.CONFIG1, synth.CONFIG2])
def test_sizes_match_reference_bookkeeping(w):
    cfg = B.Config(nodes=w.nodes, max_sims=w.n_sims, time_steps=w.time_steps, bold_tr=w.bold_tr,
                   window_size=w.window_size, window_step=w.window_step, bold_remove_s=w.bold_remove_s,
                   exc_interhem=w.exc_interhem)
    s = cfg.sizes()
    assert s["frames"] == w.frames
    assert s["n_vols_remove"] == w.n_vols_remove
    assert s["corr_len"] == w.corr_len
    assert s["n_pairs"] == w.n_pairs
    assert s["n_windows"] == w.n_windows
    assert s["n_fcd"] == w.n_windows * (w.n_windows - 1) // 2
    assert s["noise_len"] == w.nodes * (w.time_steps + 1) * 20


def test_known_reference_sizes():
    # example/run_CMAES.sh: 60 s at TR 1 s, window 10 step 2, 100 nodes -> 2450 FC, 55 FCD
    s = B.Config(nodes=100, time_steps=60000, bold_tr=1000, window_size=10, window_step=2).sizes()
    assert (s["frames"], s["corr_len"], s["n_pairs"], s["n_windows"], s["n_fcd"]) == (61, 31, 2450, 11, 55)
    ref_fc = os.path.join(ROOT, "tests", "golden")  # noqa: F841  (sizes pinned against the example files' lengths)
    s1 = B.Config(nodes=100, time_steps=450000, bold_tr=720, window_size=44, window_step=1).sizes()
    assert (s1["frames"], s1["n_windows"], s1["n_fcd"]) == (626, 541, 146070)


@pytest.mark.parametrize("kw,msg", [
    (dict(nodes=11), "even"),                                    # exc_interhem needs an even split
    (dict(time_steps=20000, bold_tr=1000), "frames"),            # 21 frames, 30 removed
    (dict(time_steps=40000, window_size=44), "windows"),         # no FCD window fits
    (dict(nodes=1), "nodes"),
    (dict(window_step=0), "window_step"),
])
def test_bad_configurations_are_status_codes(kw, msg):
    cfg = B.Config(**{**dict(nodes=10, time_steps=60000, bold_tr=1000, window_size=4), **kw})
    with pytest.raises(B.BnmError) as e:
        cfg.sizes()
    assert e.value.code == B.BNM_EINVAL
    assert msg in str(e.value)


def test_env_configuration_like_the_reference():
    code = ("import bnm_cuda_b200 as B; c = B.Config.from_env(); "
            "print(c.bold_remove_s, c.init_delta, c.exc_interhem, c.max_fic_trials, c.fic_penalty_scale)")
    env = dict(os.environ, BNM_BOLD_REMOVE="7", BNM_INIT_DELTA="0.03", BNM_EXC_INTERHEM="0",
               BNM_MAX_FIC_TRIALS_CMAES="4", BNM_CMAES_FIC_PENALTY_SCALE="1.5", PYTHONPATH=ROOT)
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, cwd=ROOT)
    vals = out.stdout.split()
    assert vals[0] == "7" and vals[2] == "0" and vals[3] == "4"
    assert float(vals[1]) == float(np.float32(0.03))  # doubles pass through float (helpers.cpp:4-11)
    assert float(vals[4]) == 1.5


def test_gram_arithmetic_defaults_to_auto():
    """The C default (bnm_config_default) and the Python default agree: the
    Gram arithmetic is chosen by precision when the plan is made (split BF16
    tensor-core Grams for the FP32 path, FP32 / FP64 SIMT analysis for the
    reference-order precisions)."""
    assert B.Config().gram == B.GRAM_AUTO
    assert B.Config.from_env().gram == B.GRAM_AUTO
    for g in (B.GRAM_AUTO, B.GRAM_F32, B.GRAM_BF16, B.GRAM_BF16_SPLIT):  # accepted by the size check
        B.Config(nodes=10, time_steps=60000, bold_tr=1000, window_size=4, gram=g).sizes()


def test_no_device_is_an_error_not_a_crash():
    if B.lib().bnm_device_count() > 0:
        pytest.skip("a GPU is present")
    cfg = B.Config(nodes=10, max_sims=2, time_steps=12000, bold_tr=1000, window_size=4, window_step=1,
                   bold_remove_s=2)
    s = cfg.sizes()
    with pytest.raises(B.BnmError) as e:
        B.Plan(cfg, synth.make_sc(10, 0.5, 0), np.zeros(s["n_pairs"]), np.zeros(s["n_fcd"]))
    assert e.value.code in (B.BNM_ECUDA, B.BNM_ENOMEM)


# ------------------------------------------------------------- CMA-ES
def _objective(X):
    D = X.shape[0]
    t = np.linspace(0.2, 0.8, D)[:, None]
    return ((X - t) ** 2).sum(0) + 0.05 * np.sin(7 * X).sum(0)


@pytest.mark.parametrize("name", ["cmaes_l10_d3_v6", "cmaes_l16_d9_v16"])
def test_cmaes_reproduces_reference_bit_for_bit(name, golden):
    g = golden[name]
    lam, dim, seed, it_max, var = [int(v) for v in g["meta"]]
    c = B.CMAES(lam, dim, seed, it_max, from_env=False, variante=var)
    for gen in range(len(g["feas"])):
        feas, _, _ = c.samples()
        np.testing.assert_array_equal(feas, g["feas"][gen])
        _, pen = c.tell(_objective(feas))
        np.testing.assert_array_equal(pen, g["penalized"][gen])
    x, v = c.best()
    np.testing.assert_array_equal(x, g["best"][:dim])
    assert v == g["best"][dim]
    assert c.iteration >= it_max


@pytest.mark.parametrize("variante", [6, 16])
def test_cmaes_checkpoint_resumes_bit_for_bit(variante, tmp_path):
    """bnm_cmaes_save after generation 5, bnm_cmaes_load into a new optimiser:
    the resumed run samples, penalises and keeps its best exactly as the
    uninterrupted one through generation 11."""
    def cost(x):  # [dim][lambda] -> [lambda]
        return ((x - 0.3) ** 2).sum(0) + 0.01 * np.sin(13 * x).sum(0)

    path = str(tmp_path / "cmaes.ckpt")
    a = B.CMAES(16, 3, 5, 40, from_env=False, variante=variante)
    hist = []
    for g in range(12):
        f, r, p = a.samples()
        it, pen = a.tell(cost(f))
        hist.append((f, r, p, it, pen, *a.best(), *a.state()))
        if g == 5:
            a.save(path)
            assert not os.path.exists(path + ".tmp")
    b = B.CMAES.load(path)
    assert (b.lam, b.dim, b.it_max) == (16, 3, 40)
    assert b.iteration == hist[5][3]
    for g in range(6, 12):
        f, r, p = b.samples()
        it, pen = b.tell(cost(f))
        got = (f, r, p, it, pen, *b.best(), *b.state())
        for x, y in zip(got, hist[g]):
            np.testing.assert_array_equal(x, y)


def test_cmaes_checkpoint_rejects_other_files(tmp_path):
    a = B.CMAES(8, 2, 1, 10, from_env=False)
    good = str(tmp_path / "good.ckpt")
    a.save(good)
    data = open(good, "rb").read()
    for name, content in (("short", data[:-8]), ("long", data + b"\0"), ("magic", b"X" + data[1:])):
        bad = str(tmp_path / name)
        open(bad, "wb").write(content)
        with pytest.raises(B.BnmError):
            B.CMAES.load(bad)
    with pytest.raises(B.BnmError):
        B.CMAES.load(str(tmp_path / "missing.ckpt"))
    with pytest.raises(B.BnmError):
        a.save(str(tmp_path / "no" / "such" / "dir.ckpt"))


def test_cmaes_cancels_on_a_covariance_that_is_not_positive(tmp_path):
    """Host-side fault injection through the checkpoint format: a saved state
    whose covariance has a negative diagonal entry makes the next
    bnm_cmaes_tell stop the run (iteration = it_max, as the reference's
    CMAES_Points cancels, cmaes.cpp:402-420) instead of sampling from it."""
    import ctypes

    a = B.CMAES(8, 2, 3, 30, from_env=False)
    for _ in range(3):
        f, _, _ = a.samples()
        a.tell(((f - 0.4) ** 2).sum(0))
    path = tmp_path / "ok.ckpt"
    a.save(str(path))
    data = bytearray(path.read_bytes())
    # magic (8 bytes), version (4), the parameter struct, 4 ints, 10 doubles,
    # 4 ints, then length-prefixed vectors; the covariance C is the 22nd
    off = 8 + 4 + ctypes.sizeof(B._CmaesParams) + 16 + 80 + 16
    for _ in range(21):
        n = int.from_bytes(data[off:off + 8], "little")
        off += 8 + 8 * n
    assert int.from_bytes(data[off:off + 8], "little") == 4  # D x D
    data[off + 8:off + 16] = np.float64(-1.0).tobytes()  # C[0][0]
    bad = tmp_path / "bad.ckpt"
    bad.write_bytes(bytes(data))
    b = B.CMAES.load(str(bad))
    f, _, _ = b.samples()
    it, _ = b.tell(((f - 0.4) ** 2).sum(0))
    assert it == 30
