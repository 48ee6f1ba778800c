"""The drop-in CLI (bnm_cuda_b200/run_CMAES_gpu) on a small synthetic case:
same arguments as the reference's run_CMAES (run_CMAES.cpp:192-218), same
output directories, log lines and best-simulation files (bnm.cu:771-833)."""
import json
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
CLI = os.path.join(ROOT, "bnm_cuda_b200", "run_CMAES_gpu")


def test_cli_usage_without_gpu():
    out = subprocess.run([CLI], capture_output=True, text=True)
    assert out.returncode == 0 and out.stdout.startswith("Usage: ./run_CMAES_")


@pytest.mark.gpu
@pytest.mark.parametrize("het", ["none", "wee-wei"])
def test_cli_runs_cmaes_and_writes_reference_files(tmp_path, golden, het):
    g = golden["n10_t12s"]
    N, T, TR, ws, step, remove, exc, nvr, seed = [int(v) for v in g["meta"]]
    d = tmp_path / "sub-01"
    d.mkdir()
    np.savetxt(d / "SC.txt", g["sc"])
    np.savetxt(d / "sub-01_desc-FCtril.txt", g["emp_fc"])
    np.savetxt(d / "sub-01_desc-FCDtril.txt", g["emp_fcd"])
    np.savetxt(d / "maps.txt", np.random.default_rng(0).standard_normal((2, N)))
    lam, it_max = 6, 3
    args = [CLI, str(d / "SC.txt"), "same", str(d / "sub-01_desc-FCtril.txt"), str(d / "sub-01_desc-FCDtril.txt"),
            str(d / "maps.txt"), str(N), "0.5-3.5", "0.05-0.5", "0.05-0.5", "0", het, str(T), str(TR), str(step),
            str(ws), "410", str(lam), str(it_max), "1"]
    env = dict(os.environ, BNM_BOLD_REMOVE=str(remove))
    r = subprocess.run(args, capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stderr + r.stdout
    multi = "_multimaps" if het != "none" else ""
    cm, sims = d / "SC" / f"cmaes{multi}_gpu", d / "SC" / f"sims{multi}_gpu"
    logs = list(cm.iterdir())
    assert len(logs) == 1
    name = logs[0].name
    assert name.startswith("sub-01_G_0.5-3.5_wee_0.05-0.5_wei_0.05-0.5_wie_0_het-" + het)
    assert name.endswith(f"_SeedMW-1_SeedSim-410_n-{it_max}x{lam}.txt")
    log = logs[0].read_text()
    dim = 3 + (2 * 2 if het != "none" else 0)
    assert log.startswith(f"Running {dim}D CMAES\nSC: ")
    assert "Free parameters: G (0.500000-3.500000) " in log
    assert len(re.findall(r"^Iteration \d+$", log, re.M)) == it_max - 1
    rows = re.findall(r"^\t IndPar \d+: .*gof=(-?[\d.]+),fic_penalty=([\d.]+),penalized_cost=([\d.]+)$", log, re.M)
    assert len(rows) == lam * (it_max - 1)
    assert re.search(r"^Best feasible parameters: G=.*gof=-?[\d.]+,fic_penalty=[\d.]+,gof_fic_penalty=-?[\d.]+$",
                     log, re.M)
    prefix = name[:-4] + "_"
    bold = np.loadtxt(sims / (prefix + "bold.txt"))
    assert bold.shape == (T // TR + 1, N)
    for f in ["S_E", "I_E", "r_E", "S_I", "I_I", "r_I", "w_EE", "w_EI", "w_IE"]:
        assert np.loadtxt(sims / (prefix + f + ".txt")).shape == (N,)
    assert (sims / (prefix + "fic_ntrials.txt")).read_text().endswith("of max 10")
    assert (sims / (prefix + "fic_failed.txt")).read_text() in ("0", "1")


@pytest.mark.gpu
def test_cli_checkpoint_resume_gives_the_uninterrupted_run(tmp_path, golden):
    """BNM_B200_CHECKPOINT: a run stopped after two generations
    (BNM_B200_MAX_GENERATIONS=2, exit status 75) and started again with the
    same checkpoint writes the same log and best-simulation files as a run
    that was never interrupted."""
    g = golden["n10_t12s"]
    N, T, TR, ws, step, remove, exc, nvr, seed = [int(v) for v in g["meta"]]
    lam, it_max = 6, 5

    def setup(name):
        d = tmp_path / name / "sub-01"
        d.mkdir(parents=True)
        np.savetxt(d / "SC.txt", g["sc"])
        np.savetxt(d / "sub-01_desc-FCtril.txt", g["emp_fc"])
        np.savetxt(d / "sub-01_desc-FCDtril.txt", g["emp_fcd"])
        args = [CLI, str(d / "SC.txt"), "same", str(d / "sub-01_desc-FCtril.txt"),
                str(d / "sub-01_desc-FCDtril.txt"), "none", str(N), "0.5-3.5", "0.05-0.5", "0.05-0.5", "0", "none",
                str(T), str(TR), str(step), str(ws), "410", str(lam), str(it_max), "1"]
        return d, args

    env = dict(os.environ, BNM_BOLD_REMOVE=str(remove))
    da, args = setup("straight")
    metrics = tmp_path / "metrics.jsonl"
    r = subprocess.run(args, capture_output=True, text=True, env=dict(env, BNM_B200_METRICS=str(metrics)),
                       timeout=600)
    assert r.returncode == 0, r.stderr + r.stdout
    lines = [json.loads(x) for x in metrics.read_text().splitlines()]  # BNM_B200_METRICS: one line per generation
    assert [m["iteration"] for m in lines] == list(range(1, it_max))
    for m in lines:
        assert m["simulations"] == lam and m["sims_per_s"] > 0 and m["device_ms"]["total"] > 0
        assert np.isfinite(m["best_gof"]) and np.isfinite(m["generation_best_cost"])
    db, args = setup("resumed")
    ck = str(tmp_path / "resumed" / "run.ckpt")
    r = subprocess.run(args, capture_output=True, text=True, env=dict(env, BNM_B200_CHECKPOINT=ck,
                                                                      BNM_B200_MAX_GENERATIONS="2"), timeout=600)
    assert r.returncode == 75, r.stderr + r.stdout
    assert os.path.exists(ck) and "Stopped after 2 generations" in r.stdout
    r = subprocess.run(args, capture_output=True, text=True, env=dict(env, BNM_B200_CHECKPOINT=ck), timeout=600)
    assert r.returncode == 0, r.stderr + r.stdout
    assert "Resuming from" in r.stdout
    for sub in ("cmaes_gpu", "sims_gpu"):
        fa, fb = sorted((da / "SC" / sub).iterdir()), sorted((db / "SC" / sub).iterdir())
        assert [f.name for f in fa] == [f.name for f in fb] and fa
        for x, y in zip(fa, fb):
            assert x.read_text().replace(str(da), str(db)) == y.read_text(), x.name
