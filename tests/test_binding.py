"""The reference's own driver on this library.

oracle/_ref/run_CMAES_refdrv is the reference's run_CMAES.cpp, unmodified,
compiled as its GPU build does (nvcc) with bnm_cuda_b200/binding/bnm.cu in
place of the reference's bnm.cu (oracle/Makefile, target refdrv): every
run_simulations call of the driver (run_CMAES.cpp:758-780 per generation,
875-897 for the best particle) goes through the C ABI.  The driver computes
analytic FIC on the host (fic.cpp) and passes its host noise stream; the
binding derives the window step from the driver's window table.

On the same command line and seeds it must produce what this library's own
drop-in driver (bnm_cuda_b200/run_CMAES_gpu) produces: the same CMA-ES log
(every generation's parameters, gof, FIC penalty and penalised cost; the best
point) and the same best-simulation files, up to the printed precision.  The
two differ only where the analytic FIC runs (host FP64 Brent vs the device's),
which agree to 1e-10.  Run for the FP32 product path and the FP64
reference-order path, with a window step of 2 so that the step really is read
from the driver's table.
"""
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
CLI = os.path.join(ROOT, "bnm_cuda_b200", "run_CMAES_gpu")
REFDRV = os.path.join(ROOT, "oracle", "_ref", "run_CMAES_refdrv")
NUM = re.compile(r"-?\d+\.\d+(?:e[-+]\d+)?|-?\d+")


def _run(exe, d, g, het, step, env):
    N, T, TR, ws, _, remove, exc, nvr, seed = [int(v) for v in g["meta"]]
    lam, it_max = 6, 4
    args = [exe, str(d / "SC.txt"), "same", str(d / "sub-01_desc-FCtril.txt"), str(d / "sub-01_desc-FCDtril.txt"),
            str(d / "maps.txt"), str(N), "0.5-3.5", "0.05-0.5", "0.05-0.5", "0", het, str(T), str(TR), str(step),
            str(ws), "410", str(lam), str(it_max), "1"]
    r = subprocess.run(args, capture_output=True, text=True, env=env, timeout=900)
    assert r.returncode == 0, (exe, r.stderr[-2000:], r.stdout[-2000:])
    multi = "_multimaps" if het != "none" else ""
    logs = list((d / "SC" / f"cmaes{multi}_gpu").iterdir())
    assert len(logs) == 1
    return logs[0], d / "SC" / f"sims{multi}_gpu"


def _case_dir(root, g, step):
    N, T, TR, ws, _, remove, exc, nvr, seed = [int(v) for v in g["meta"]]
    root.mkdir()
    np.savetxt(root / "SC.txt", g["sc"])
    np.savetxt(root / "sub-01_desc-FCtril.txt", g["emp_fc"])
    np.savetxt(root / "sub-01_desc-FCDtril.txt", np.random.default_rng(step).uniform(-0.3, 1.0, 300))
    np.savetxt(root / "maps.txt", np.random.default_rng(0).standard_normal((2, N)))
    return root


def _compare_text(a, b, atol):
    la, lb = a.splitlines(), b.splitlines()
    assert len(la) == len(lb), (len(la), len(lb))
    for x, y in zip(la, lb):
        if x.startswith(("SC: ", "FC: ", "Maps: ")):  # input paths
            continue
        assert NUM.sub("#", x) == NUM.sub("#", y), (x, y)
        u = np.array([float(v) for v in NUM.findall(x)])
        w = np.array([float(v) for v in NUM.findall(y)])
        np.testing.assert_allclose(u, w, atol=atol, rtol=0, err_msg=f"{x}\n{y}")


def test_reference_driver_was_built_against_the_library():
    if not os.path.exists(REFDRV):
        pytest.skip("reference driver not built (make -C oracle refdrv needs the reference sources)")
    out = subprocess.run(["nm", "-D", "--undefined-only", REFDRV], capture_output=True, text=True).stdout
    for sym in ("bnm_plan_create", "bnm_run", "bnm_config_sizes"):
        assert re.search(rf"\bU {sym}\b", out), sym


@pytest.mark.gpu
@pytest.mark.parametrize("precision,het,atol", [("f32", "none", 2e-5), ("f64", "wee-wei", 2e-6)])
def test_reference_driver_on_the_library_matches_the_drop_in_cli(tmp_path, golden, precision, het, atol):
    if not os.path.exists(REFDRV):
        pytest.skip("reference driver not built")
    g = golden["n10_t12s"]
    remove = int(g["meta"][5])
    step = 2
    env = dict(os.environ, BNM_BOLD_REMOVE=str(remove), BNM_B200_PRECISION=precision)
    log_ref, sims_ref = _run(REFDRV, _case_dir(tmp_path / "a", g, step), g, het, step, env)
    log_cli, sims_cli = _run(CLI, _case_dir(tmp_path / "b", g, step), g, het, step, env)
    assert log_ref.name == log_cli.name
    _compare_text(log_ref.read_text(), log_cli.read_text(), atol)
    files = sorted(p.name for p in sims_ref.iterdir())
    assert files == sorted(p.name for p in sims_cli.iterdir())
    assert any(f.endswith("_bold.txt") for f in files) and any(f.endswith("_fic_ntrials.txt") for f in files)
    for f in files:
        _compare_text((sims_ref / f).read_text(), (sims_cli / f).read_text(), atol)
