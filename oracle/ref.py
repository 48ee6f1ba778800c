"""TEST INFRASTRUCTURE ONLY (oracle): ctypes access to

* ``_ref/libbnmref_{f64,f32}.so`` -- the reference's own CPU sources
  (bnm.cpp, check_fit.cpp, fic.cpp, cmaes.cpp) compiled unmodified against the
  GSL/libks stand-ins in ``compat/`` (see Makefile), and
* ``libbnm_port.so`` -- this project's CPU restatement of the same path
  (bnm_port.cpp), which the tests pin against the reference build and then
  use to check the CUDA path.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this module.  The reference reads its ``BNM_*`` configuration from the
environment when the library is loaded (constants.h:93-116), so callers that
need another configuration run in a fresh process (``run_isolated``).
"""
from __future__ import annotations

import ctypes as C
import os
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_libs: dict = {}

dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def ref_available(fp32: bool = False) -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", f"libbnmref_{'f32' if fp32 else 'f64'}.so"))


def port_available() -> bool:
    return os.path.exists(os.path.join(HERE, "libbnm_port.so"))


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def ref_lib(fp32: bool = False):
    key = "f32" if fp32 else "f64"
    if key not in _libs:
        lib = C.CDLL(os.path.join(HERE, "_ref", f"libbnmref_{key}.so"))
        lib.ref_run_simulations.argtypes = [dp, dp, dp, dp, dp, dp, dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                            C.c_int, C.c_int, dp, C.c_int, dp, C.c_int, C.c_int, C.c_int, C.c_int,
                                            C.c_int, C.c_char_p, C.c_int, C.c_int, C.c_int]
        lib.ref_fc_tril.argtypes = [dp, C.c_int, C.c_int, C.c_int, dp]
        lib.ref_fcd_tril.argtypes = [dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, dp, C.c_int]
        lib.ref_check_fit_bold.argtypes = [dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, dp, C.c_int, dp, C.c_int,
                                           C.c_int, C.c_int]
        lib.ref_check_fit_bold.restype = C.c_double
        lib.ref_ks_stat.argtypes = [dp, C.c_int, dp, C.c_int]
        lib.ref_ks_stat.restype = C.c_double
        lib.ref_analytical_fic.argtypes = [dp, C.c_int, C.c_double, dp, dp, dp]
        lib.ref_constants.argtypes = [dp]
        lib.ref_cmaes_setup.argtypes = [C.c_int] * 4
        lib.ref_cmaes_get.argtypes = [dp, dp, dp]
        lib.ref_cmaes_tell.argtypes = [dp, dp]
        lib.ref_cmaes_best.argtypes = [dp]
        lib.ref_cmaes_state.argtypes = [dp, dp, dp]
        lib.ref_calculate_params.argtypes = [C.c_int, C.c_int, C.c_int, dp, C.c_double, C.c_double, C.c_double,
                                             C.c_double, dp, dp, dp, dp, dp]
        lib.ref_run_cmaes_cpu.argtypes = [C.c_int, C.POINTER(C.c_char_p)]
        lib.ref_run_particles_timed.argtypes = [dp, dp, dp, dp, dp, dp, dp, C.c_int, C.c_int, C.c_int, C.c_int,
                                                C.c_int, C.c_int, dp, C.c_int, dp, C.c_int, C.c_int, C.c_int,
                                                C.c_int, C.c_char_p, dp]
        _libs[key] = lib
    return _libs[key]


def port_lib():
    if "port" not in _libs:
        lib = C.CDLL(os.path.join(HERE, "libbnm_port.so"))
        lib.port_noise.argtypes = [C.c_int, C.c_int64, fp]
        lib.port_analytic_fic.argtypes = [C.c_int, dp, C.c_int, C.c_double, dp, dp, dp]
        integ = [dp, C.c_int, C.c_double, dp, dp, dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p,
                 C.c_int, C.c_int, C.c_double, dp, dp, C.POINTER(C.c_int), C.POINTER(C.c_int), dp]
        lib.port_integrate_f64.argtypes = integ
        lib.port_integrate_f32.argtypes = integ
        lib.port_fic_penalty.argtypes = [C.c_int, dp, C.c_int, C.c_double, C.c_int, C.c_int]
        lib.port_fic_penalty.restype = C.c_double
        lib.port_fc_tril.argtypes = [dp, C.c_int, C.c_int, C.c_int, dp]
        lib.port_windows.argtypes = [C.c_int, C.c_int, C.c_int, ip, ip, C.c_int]
        lib.port_fcd_tril.argtypes = [dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, dp, C.c_void_p]
        lib.port_gof.argtypes = [dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, dp, C.c_int, dp, C.c_int, C.c_int,
                                 C.c_double, dp]
        lib.port_ks.argtypes = [dp, C.c_int, dp, C.c_int]
        lib.port_ks.restype = C.c_double
        lib.port_run_batch.argtypes = [C.c_int, C.c_int, dp, C.c_int, dp, dp, dp, dp, C.c_int, C.c_int, C.c_int,
                                       C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_double,
                                       C.c_int, C.c_int, C.c_int, dp, C.c_int, dp, C.c_int, C.c_int, C.c_double,
                                       C.c_double, C.c_int, C.c_int, dp, dp, dp, ip, ip]
        _libs["port"] = lib
    return _libs["port"]


# --------------------------------------------------------------- reference
def ref_constants(fp32=False) -> dict:
    out = np.zeros(15)
    ref_lib(fp32).ref_constants(out)
    keys = ["bold_remove_s", "max_cost", "i_sampling_start", "i_sampling_end", "i_sampling_duration",
            "numerical_fic", "max_fic_trials_cmaes", "init_delta", "use_fc_diff", "exc_interhem",
            "fic_penalty_scale", "fic_reject_failed", "sigma", "early_stop_gens", "early_stop_tol"]
    return dict(zip(keys, out.tolist()))


def ref_run_simulations(SC, G, wEE, wEI, wIE, *, time_steps, bold_tr, rand_seed, max_fic_trials, emp_fc, emp_fcd,
                        window_step, window_size, calculate_fic_penalty=True, sim_only=False, no_fcd=False,
                        out_prefix="", save_output=False, extended_output=False, fp32=False):
    """run_simulations of bnm.cpp:431-466.  Returns (cost[n], fic_penalty[n])."""
    n, N = len(G), SC.shape[0]
    cost, pen = np.zeros(n), np.zeros(n)
    emp_fcd = _d(emp_fcd) if emp_fcd is not None and len(emp_fcd) else np.zeros(1)
    ref_lib(fp32).ref_run_simulations(cost, pen, _d(G), _d(wEE).ravel(), _d(wEI).ravel(), _d(wIE).ravel(), _d(SC),
                                      N, n, int(calculate_fic_penalty), time_steps, bold_tr, rand_seed,
                                      max_fic_trials, _d(emp_fc), len(emp_fc), emp_fcd, len(emp_fcd), int(sim_only),
                                      int(no_fcd), window_step, window_size, out_prefix.encode(), 0,
                                      int(save_output), int(extended_output))
    return cost, pen


def ref_run_particles_timed(SC, G, wEE, wEI, wIE, *, time_steps, bold_tr, rand_seed, max_fic_trials, emp_fc,
                            emp_fcd, window_step, window_size, out_dir="", sim_only=False, fp32=False):
    """The reference's run_simulations loop (bnm.cpp:441-465), one bnm() per
    particle under OpenMP, timed per particle.  With out_dir, each particle's
    save_output files go to <out_dir>/p<i>_* and the reference's own FIC trial
    counts are read back from them.  -> dict(cost, fic_penalty, seconds,
    trials or None)."""
    n, N = len(G), SC.shape[0]
    cost, pen, sec = np.zeros(n), np.zeros(n), np.zeros(n)
    ref_lib(fp32).ref_run_particles_timed(cost, pen, _d(G), _d(wEE).ravel(), _d(wEI).ravel(), _d(wIE).ravel(),
                                          _d(SC), N, n, time_steps, bold_tr, rand_seed, max_fic_trials, _d(emp_fc),
                                          len(emp_fc), _d(emp_fcd), len(emp_fcd), window_step, window_size,
                                          int(sim_only), out_dir.encode(), sec)
    trials = None
    if out_dir:
        trials = np.array([int(open(os.path.join(out_dir, f"p{i}_fic_ntrials.txt")).read().split()[0])
                           for i in range(n)])
    return dict(cost=cost, fic_penalty=pen, seconds=sec, trials=trials)


def ref_fc_tril(bold, exc=True, fp32=False):
    bold = _d(bold)
    T, N = bold.shape
    out = np.zeros(N * N)
    n = ref_lib(fp32).ref_fc_tril(bold, T, N, int(exc), out)
    return None if n < 0 else out[:n]


def ref_fcd_tril(bold, step, window_size, exc=True, drop_edges=True, fp32=False):
    bold = _d(bold)
    T, N = bold.shape
    cap = T * T
    out = np.zeros(cap)
    n = ref_lib(fp32).ref_fcd_tril(bold, T, N, step, window_size, int(drop_edges), int(exc), out, cap)
    return None if n < 0 else out[:n]


def ref_check_fit_bold(bold, step, window_size, emp_fc, emp_fcd, exc=True, no_fcd=False, fp32=False):
    bold = _d(bold)
    T, N = bold.shape
    return ref_lib(fp32).ref_check_fit_bold(bold, T, N, step, window_size, 1, _d(emp_fc), len(emp_fc), _d(emp_fcd),
                                            len(emp_fcd), int(no_fcd), int(exc))


def ref_analytical_fic(SC, G, wEE, wEI, fp32=False):
    N = SC.shape[0]
    out = np.zeros(N)
    unstable = ref_lib(fp32).ref_analytical_fic(_d(SC), N, float(G), _d(wEE), _d(wEI), out)
    return out, bool(unstable)


def ref_calculate_params(nodes, het_mask, maps, G, wee, wie, wei, scales, fp32=False):
    """calculate_params of run_CMAES.cpp:61-143 for one particle.
    -> (G, wEE [N], wEI [N], wIE [N])."""
    maps = _d(np.zeros((0, nodes)) if maps is None else maps).reshape(-1, nodes)
    scales = _d(np.zeros((3, max(len(maps), 1))) if scales is None else scales)
    g, ee, ei, ie = np.zeros(1), np.zeros(nodes), np.zeros(nodes), np.zeros(nodes)
    ref_lib(fp32).ref_calculate_params(nodes, het_mask, len(maps), maps if len(maps) else np.zeros(1), G, wee, wie,
                                       wei, scales, g, ee, ei, ie)
    return g[0], ee, ei, ie


# -------------------------------------------------------------------- port
def port_noise(seed: int, n: int) -> np.ndarray:
    out = np.zeros(n, dtype=np.float32)
    port_lib().port_noise(seed, n, out)
    return out


def port_analytic_fic(SC, G, wEE, wEI, fp32=False):
    N = SC.shape[0]
    out = np.zeros(N)
    u = port_lib().port_analytic_fic(int(fp32), _d(SC), N, float(G), _d(wEE), _d(wEI), out)
    return out, bool(u)


def port_integrate(SC, G, wEE, wEI, wIE, *, time_steps, bold_tr, n_vols_remove, seed=0, noise=None,
                   adjust_fic=True, max_fic_trials=10, sampling_start=1000, sampling_end=10000,
                   init_delta=float(np.float32(0.02)), fp32=False):
    """One simulation of bnm.cpp:26-290.  Returns dict(bold [frames, N],
    wIE [N], trials, failed, ext [6, N] = means of S_E, I_E, r_E, S_I, I_I, r_I)."""
    N = SC.shape[0]
    frames = time_steps // bold_tr + 1
    bold, w, ext = np.zeros(frames * N), np.zeros(N), np.zeros(6 * N)
    tr, fl = C.c_int(0), C.c_int(0)
    nz = None
    if noise is not None:
        noise = np.ascontiguousarray(noise, dtype=np.float32)
        nz = noise.ctypes.data_as(C.c_void_p)
    fn = port_lib().port_integrate_f32 if fp32 else port_lib().port_integrate_f64
    fn(_d(SC), N, float(G), _d(wEE), _d(wEI), _d(wIE), int(adjust_fic), max_fic_trials, time_steps, bold_tr,
       n_vols_remove, seed, nz, sampling_start, sampling_end, init_delta, bold, w, C.byref(tr), C.byref(fl), ext)
    return dict(bold=bold.reshape(frames, N), wIE=w, trials=tr.value, failed=fl.value, ext=ext.reshape(6, N))


def port_fic_penalty(mean_rE, failed=0, scale=2.0, reject_failed=0, fp32=False):
    mean_rE = _d(mean_rE)
    return port_lib().port_fic_penalty(int(fp32), mean_rE, len(mean_rE), scale, reject_failed, int(failed))


def port_fc_tril(bold, exc=True):
    bold = _d(bold)
    T, N = bold.shape
    out = np.zeros(N * N)
    n = port_lib().port_fc_tril(bold, T, N, int(exc), out)
    return None if n < 0 else out[:n]


def port_fcd_tril(bold, step, window_size, exc=True, window_fc=False):
    bold = _d(bold)
    T, N = bold.shape
    out = np.zeros(T * T)
    P = N * (N - 1) // 2 - ((N // 2) ** 2 if exc else 0)
    wfc = np.zeros(T * P) if window_fc else None
    n = port_lib().port_fcd_tril(bold, T, N, step, window_size, int(exc), out,
                                 wfc.ctypes.data_as(C.c_void_p) if window_fc else None)
    if n < 0:
        return None
    if window_fc:
        W = int(round((1 + np.sqrt(1 + 8 * n)) / 2))
        return out[:n], wfc[:W * P].reshape(W, P)
    return out[:n]


def port_gof(bold, step, window_size, emp_fc, emp_fcd, exc=True, use_fc_diff=True, max_cost=2.0):
    """-> dict(fc_corr, fc_diff, fcd_ks, cost) of check_fit.cpp:138-217."""
    bold = _d(bold)
    T, N = bold.shape
    out = np.zeros(4)
    port_lib().port_gof(bold, T, N, step, window_size, int(exc), _d(emp_fc), len(emp_fc), _d(emp_fcd), len(emp_fcd),
                        int(use_fc_diff), max_cost, out)
    return dict(fc_corr=out[0], fc_diff=out[1], fcd_ks=out[2], cost=out[3])


def port_ks(x, y):
    return port_lib().port_ks(_d(x), len(x), _d(y), len(y))


def port_run_batch(SC, G, wEE, wEI, wIE, *, time_steps, bold_tr, n_vols_remove, seed, window_step, window_size,
                   emp_fc, emp_fcd, noise=None, do_fic=True, adjust_fic=True, max_fic_trials=10, exc=True,
                   use_fc_diff=True, max_cost=2.0, pen_scale=2.0, reject_failed=0, sampling_start=1000,
                   sampling_end=10000, init_delta=float(np.float32(0.02)), fp32=False, n_threads=0):
    """OpenMP batch of port simulations.  -> dict(cost, fic_penalty, wIE, trials, failed)."""
    n, N = len(G), SC.shape[0]
    cost, pen, w = np.zeros(n), np.zeros(n), np.zeros(n * N)
    tr, fl = np.zeros(n, np.int32), np.zeros(n, np.int32)
    nz = None
    if noise is not None:
        noise = np.ascontiguousarray(noise, dtype=np.float32)
        nz = noise.ctypes.data_as(C.c_void_p)
    port_lib().port_run_batch(int(fp32), n, _d(SC), N, _d(G), _d(wEE).ravel(), _d(wEI).ravel(), _d(wIE).ravel(),
                              int(do_fic), int(adjust_fic), max_fic_trials, time_steps, bold_tr, n_vols_remove, seed,
                              nz, sampling_start, sampling_end, init_delta, window_step, window_size, int(exc),
                              _d(emp_fc), len(emp_fc), _d(emp_fcd), len(emp_fcd), int(use_fc_diff), max_cost,
                              pen_scale, reject_failed, n_threads, cost, pen, w, tr, fl)
    return dict(cost=cost, fic_penalty=pen, wIE=w.reshape(n, N), trials=tr, failed=fl)


def run_isolated(fn, *args, env=None, **kwargs):
    """Run ``fn`` in a fresh spawned process with extra environment (the
    reference reads BNM_* at load time)."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    with ctx.Pool(1, initializer=_set_env, initargs=(env or {},)) as pool:
        return pool.apply(fn, args, kwargs)


def _set_env(env):
    os.environ.update({k: str(v) for k, v in env.items()})


def port_final_pass(SC, G, wEE, wEI, wIE_final, *, time_steps, bold_tr, n_vols_remove, step, window_size, emp_fc,
                    emp_fcd, exc=True, seed=410, noise=None, fp32=False):
    """The final pass of one simulation, recomputed from its final wIE.

    After the last FIC decision (bnm.cpp:230-289) a simulation either restarts
    from t = 0 with the adjusted wIE or continues; either way the BOLD it
    reports comes from one uninterrupted pass from t = 0 with the final wIE and
    the noise stream from its start (the stream restarts with every trial,
    bnm.cpp:273-274).  So a simulation whose FIC decisions differ from the
    oracle's (a node's mean current on the threshold can flip under last-ulp
    differences) is still checked: this reruns the port with numerical FIC off
    and wIE = the simulation's own final wIE, and returns its BOLD, FC, FCD
    and goodness of fit (check_fit.cpp:138-217, FP64)."""
    r = port_integrate(SC, G, wEE, wEI, np.asarray(wIE_final, np.float64), time_steps=time_steps, bold_tr=bold_tr,
                       n_vols_remove=n_vols_remove, seed=seed, noise=noise, adjust_fic=False, fp32=fp32)
    kept = r["bold"][n_vols_remove:]
    fit = port_gof(kept, step, window_size, emp_fc, emp_fcd, exc=exc)
    return dict(bold=r["bold"], fc=port_fc_tril(kept, exc), fcd=port_fcd_tril(kept, step, window_size, exc),
                cost=fit["cost"], ext=r["ext"])


def every_particle_reference(dev, ref, trials_ref, wie_ref, *, floor, rerun):
    """Reference values for every particle of a device batch.

    dev: the device's outputs (fic_ntrials, w_ie); ref: dict of per-particle
    reference arrays (bold, fc, fcd, cost, ...) from the oracle's own FIC path.
    Particles whose FIC took the oracle's decisions (same trial count, final
    wIE equal up to FP32 rounding) keep those; every other particle gets
    rerun(i, final_wIE) (port_final_pass).  At least `floor` of the particles
    must take the oracle's decisions.  Returns (reference dict, mask of the
    particles that took the oracle's decisions)."""
    same = (np.asarray(dev["fic_ntrials"]) == np.asarray(trials_ref)) & \
        (np.abs(np.asarray(dev["w_ie"]) - np.asarray(wie_ref)).max(1) < 1e-4)
    assert same.mean() >= floor, ("FIC decisions differ from the oracle's", dev["fic_ntrials"], trials_ref)
    out = {k: [np.asarray(v[i]) for i in range(len(same))] for k, v in ref.items()}
    for i in np.flatnonzero(~same):
        rr = rerun(i, np.asarray(dev["w_ie"][i]))
        for k in out:
            out[k][i] = np.asarray(rr[k])
    return {k: np.array(v) for k, v in out.items()}, same
