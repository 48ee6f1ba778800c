"""Failure detection of the bounded device waits, without a GPU fault.

The reference exits the process on any CUDA error (bnm.cu:47-67).  Here every
device wait (noise and SC bulk copies, the cluster S_E exchange, the Gram
pipeline) is bounded by wall time and reports BNM_ETIMEOUT through the plan's
status word.  The test makes one such wait run out on purpose: a kernel waits,
with the integrators' own wait routine and a 1 ms limit, on an mbarrier that
nothing arrives on (no copy or MMA is in flight), so the wait must give up.
It then checks the status code, the elapsed time, and that the device still
runs a normal batch afterwards.
"""
import numpy as np
import pytest

import bnm_cuda_b200 as B


@pytest.mark.gpu
def test_expired_wait_reports_timeout_and_device_stays_usable(golden, port):
    r = B.wait_probe(1_000_000)  # 1 ms
    assert r["code"] == B.BNM_ETIMEOUT, r
    assert r["status"] & 2, r  # kStatusTimeout
    assert 1.0 <= r["elapsed_ms"] < 200.0, r
    assert "gave up" in r["message"]
    # a zero limit gives up at the first check as well
    r0 = B.wait_probe(0)
    assert r0["code"] == B.BNM_ETIMEOUT and r0["elapsed_ms"] < 50.0, r0
    # the context is intact: a normal batch still runs and matches the oracle's FIC decisions
    g = golden["n10_t12s"]
    N, T, TR, ws, step, remove, exc, nvr, seed = [int(v) for v in g["meta"]]
    cfg = B.Config(nodes=N, max_sims=len(g["G"]), time_steps=T, bold_tr=TR, window_size=ws, window_step=step,
                   bold_remove_s=remove, exc_interhem=bool(exc), precision=B.PREC_F64, noise_mode=B.NOISE_HOST)
    with B.Plan(cfg, g["sc"], g["emp_fc"], g["emp_fcd"], host_noise=port.port_noise(410, cfg.sizes()["noise_len"])) as p:
        out = p.run(g["G"], g["wEE"], g["wEI"])
    np.testing.assert_array_equal(out["fic_ntrials"], g["ref_ntrials"])
    np.testing.assert_allclose(out["cost"], g["ref_cost_f64"], atol=1e-4)


def test_wait_probe_rejects_limits_out_of_range():
    # checked on the host before any device work (runs without a GPU)
    with pytest.raises(B.BnmError):
        B._check(B.lib().bnm_wait_probe(0, -1, None, None))
    with pytest.raises(B.BnmError):
        B._check(B.lib().bnm_wait_probe(0, 2_000_000_000, None, None))
