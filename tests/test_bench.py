"""The benchmark's reference arm on the CPU (no GPU needed): bench.py --impl
reference runs the reference's own OpenMP path (oracle/_ref) once at full
length for its value and times bounded samples as its steps.  A short
profiling case (8 particles, 80 s of model time) checks the line's contract:
one JSON line, the measured value beside the sample model, ms_per_step equal
to the samples' wall time, and the same config keys and values as the GPU
arm reports."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def test_reference_arm_line_measures_full_length_and_models_samples():
    sys.path.insert(0, ROOT)
    from oracle import ref

    if not ref.ref_available():
        pytest.skip("reference build missing (make -C oracle)")
    env = {k: v for k, v in os.environ.items() if k != "OMP_NUM_THREADS"}  # one particle per core
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--particles", "8",
                        "--model-ms", "80000", "--steps", "1", "--warmup", "0"], capture_output=True, text=True,
                       env=env, cwd=ROOT, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == "sims/s" and d["value"] > 0
    full = d["cpu_baseline"]["measured_full"]
    assert full["value"] == d["value"] and len(full["fic_restarts"]) == d["cpu_baseline"]["cores"]
    assert full["wall_s"] >= full["max_s_per_sim"] * 0.99
    assert d["cpu_baseline"]["modelled"]["value"] > 0
    assert d["ms_per_step"] > 0 and d["steps"] == 1
    assert d["e2e"] == {"value": d["value"], "unit": "sims/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    import bench

    bench.T_MS, bench.N_SIMS = 80000, 8
    bench.WORKLOAD = d["config"]["workload"]
    assert d["config"] == bench.workload_config(1)
