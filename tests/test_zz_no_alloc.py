"""bnm_gof_noalloc, the entry point for callers that cannot allocate device
memory (a host that owns the allocator, or a loop that must not call
cudaMalloc / cudaFree, whose device-wide synchronisation would stall other
streams).  Its output, computed with nothing but the library's static device
scratch array, must equal the plan path's on the same BOLD series, on two
calls in a row (the second call finds the first call's leftovers in the
shared array).  Collected last on purpose; it runs alone or after the rest."""
import numpy as np
import pytest

import bnm_cuda_b200 as B

pytestmark = pytest.mark.gpu


def test_noalloc_gof_matches_plan_twice(golden, port):
    import torch

    g = golden["n20_t25s_tr500"]
    N, T, TR, ws, step, remove, exc, nvr, seed = [int(v) for v in g["meta"]]
    cfg = B.Config(nodes=N, max_sims=len(g["G"]), time_steps=T, bold_tr=TR, window_size=ws, window_step=step,
                   bold_remove_s=remove, exc_interhem=bool(exc), noise_mode=B.NOISE_HOST,
                   gram=B.GRAM_F32)  # the allocation-free entry point runs the FP32 SIMT FCD and FP64 FC
    nz = port.port_noise(410, cfg.sizes()["noise_len"])
    with B.Plan(cfg, g["sc"], g["emp_fc"], g["emp_fcd"], host_noise=nz) as p:
        r = p.run(g["G"], g["wEE"], g["wEI"], outputs=("bold",))
    n, frames = r["bold"].shape[0], r["bold"].shape[1]
    d_bold = torch.tensor(r["bold"].astype(np.float32), device="cuda")  # the plan's own float BOLD
    d_out = torch.full((5, n), np.nan, dtype=torch.float64, device="cuda")
    for _ in range(2):
        d_out.fill_(np.nan)
        B.gof_noalloc(d_bold.data_ptr(), n, frames, N, nvr, ws, step, g["emp_fc"], g["emp_fcd"], d_out.data_ptr(),
                      exc_interhem=bool(exc))
        torch.cuda.synchronize()
        out = d_out.cpu().numpy()
        np.testing.assert_allclose(out[0], r["cost"], rtol=0, atol=1e-9)
        np.testing.assert_allclose(out[1], r["fc_corr"], rtol=0, atol=1e-9)
        np.testing.assert_allclose(out[2], r["fc_diff"], rtol=0, atol=1e-9)
        np.testing.assert_allclose(out[3], r["fcd_ks"], rtol=0, atol=1e-9)


def test_noalloc_rejects_what_does_not_fit(golden):
    import torch

    d = torch.zeros(16, device="cuda")
    out = torch.zeros(5 * 8, dtype=torch.float64, device="cuda")
    # eight N=100, 450 s / TR 0.72 s series need more than the 32 MiB scratch
    with pytest.raises(B.BnmError) as e:
        B.gof_noalloc(d.data_ptr(), 8, 626, 100, 41, 44, 1, np.zeros(2450), np.linspace(-1, 1, 146070),
                      out.data_ptr())
    assert e.value.code == B.BNM_EINVAL and "scratch" in str(e.value)
    with pytest.raises(B.BnmError) as e:
        B.lib()  # unsorted empirical FCD through the raw ABI is refused
        import ctypes as C
        efc, efcd = np.zeros(2450), np.array([0.5, 0.1, 0.3])
        rc = B.lib().bnm_gof_noalloc(C.c_void_p(d.data_ptr()), 1, 626, 100, 41, 44, 1, 1, 1, 2.0,
                                     efc.ctypes.data_as(C.c_void_p), 2450, efcd.ctypes.data_as(C.c_void_p), 3,
                                     C.c_void_p(out.data_ptr()), None)
        B._check(rc)
    assert "sorted" in str(e.value)
