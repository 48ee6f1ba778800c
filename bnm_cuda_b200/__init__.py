"""bnm_cuda_b200: B200 (sm_100a) simulate-and-fit for the reduced Wong-Wang
model with FIC, Balloon-Windkessel BOLD, FC / window FC / FCD, KS and
goodness of fit, behind the C ABI of ``include/bnm_b200.h``.

This module is the Python-side mirror of that ABI (ctypes, no torch): it
loads ``libbnm_b200.so`` built in-tree by ``bnm_cuda_b200.build`` and raises
if the library is missing -- there is no CPU fallback.

Reference correspondence (amnsbr/bnm_cuda):
    Plan.run / run_simulations -> run_simulations, bnm.cu:594-834 / bnm.cpp:431-466
    Plan.analytic_fic          -> analytical_fic, fic.cpp:130-207
    CMAES                      -> CMAES_Points, cmaes.cpp:128-557
    Config.from_env            -> BNM_* settings, constants.h:93-116
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbnm_b200.so")

BNM_OK, BNM_EINVAL, BNM_ENOMEM, BNM_ECUDA, BNM_ETIMEOUT = 0, 1, 2, 3, 4
PREC_F32, PREC_F64, PREC_F32_REF = 0, 1, 2
NOISE_PHILOX, NOISE_HOST = 0, 1
GRAM_AUTO, GRAM_F32, GRAM_BF16, GRAM_BF16_SPLIT = -1, 0, 1, 2

_lib = None


class BnmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class _Config(C.Structure):
    _fields_ = [("nodes", C.c_int32), ("max_sims", C.c_int32), ("time_steps", C.c_int32), ("bold_tr", C.c_int32),
                ("window_step", C.c_int32), ("window_size", C.c_int32), ("bold_remove_s", C.c_int32),
                ("exc_interhem", C.c_int32), ("do_fic", C.c_int32), ("numerical_fic", C.c_int32),
                ("max_fic_trials", C.c_int32), ("i_sampling_start", C.c_int32), ("i_sampling_end", C.c_int32),
                ("init_delta", C.c_double), ("use_fc_diff", C.c_int32), ("fic_reject_failed", C.c_int32),
                ("fic_penalty_scale", C.c_double), ("max_cost", C.c_double), ("calculate_fic_penalty", C.c_int32),
                ("no_fcd", C.c_int32), ("precision", C.c_int32), ("noise_mode", C.c_int32),
                ("noise_seed", C.c_uint64), ("device", C.c_int32), ("gram", C.c_int32)]


class _Sizes(C.Structure):
    _fields_ = [("frames", C.c_int32), ("n_vols_remove", C.c_int32), ("corr_len", C.c_int32),
                ("n_pairs", C.c_int32), ("n_windows", C.c_int32), ("window_len", C.c_int32), ("n_fcd", C.c_int32),
                ("noise_len", C.c_int64)]


class _BatchOut(C.Structure):
    _fields_ = [(k, C.c_void_p) for k in ("cost", "fic_penalty", "fc_corr", "fc_diff", "fcd_ks", "w_ie", "fic_failed",
                                          "fic_ntrials", "fic_unstable", "ext_means", "bold", "fc", "fcd",
                                          "fcd_left", "fcd_right")]


class _CmaesParams(C.Structure):
    _fields_ = [("lambda_", C.c_int32), ("dimension", C.c_int32), ("seed_mw", C.c_int32), ("it_max", C.c_int32),
                ("variante", C.c_int32), ("sigma", C.c_double), ("alphacov", C.c_double),
                ("gamma_scale", C.c_double), ("bound_soft_edge", C.c_double), ("early_stop_gens", C.c_int32),
                ("early_stop_tol", C.c_double)]


def lib():
    """The loaded C library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise BnmError(BNM_EINVAL, f"{LIB_PATH} is missing: run `python -m bnm_cuda_b200.build`")
        L = C.CDLL(LIB_PATH)
        vp, i32, dbl = C.c_void_p, C.c_int32, C.c_double
        L.bnm_last_error.restype = C.c_char_p
        L.bnm_config_default.argtypes = [C.POINTER(_Config)]
        L.bnm_config_from_env.argtypes = [C.POINTER(_Config)]
        L.bnm_config_sizes.argtypes = [C.POINTER(_Config), C.POINTER(_Sizes)]
        L.bnm_plan_create.argtypes = [C.POINTER(_Config), vp, vp, i32, vp, i32, vp, C.c_int64, C.POINTER(vp)]
        L.bnm_plan_destroy.argtypes = [vp]
        L.bnm_run.argtypes = [vp, i32, vp, vp, vp, vp, C.POINTER(_BatchOut)]
        L.bnm_analytic_fic.argtypes = [vp, i32, vp, vp, vp, vp, vp]
        L.bnm_last_timings.argtypes = [vp, vp]
        L.bnm_plan_integrator.argtypes = [vp, vp, vp]
        L.bnm_check_fit_bold.argtypes = [vp, i32, vp, C.POINTER(_BatchOut)]
        L.bnm_last_gram.argtypes = [vp, vp, vp]
        L.bnm_group_create.argtypes = [vp, i32, C.POINTER(vp)]
        L.bnm_group_destroy.argtypes = [vp]
        L.bnm_group_destroy.restype = None
        L.bnm_group_run.argtypes = [vp, vp, vp, vp, vp, vp]
        L.bnm_group_last.argtypes = [vp, vp, vp]
        L.bnm_plan_noise.argtypes = [vp, C.c_int64, C.c_int64, vp]
        L.bnm_measure_fp32_peak.argtypes = [i32, C.POINTER(C.c_double)]
        L.bnm_bw_math_probe.argtypes = [i32, vp, i32, vp]
        L.bnm_wait_probe.argtypes = [i32, C.c_int64, vp, vp]
        L.bnm_plan_graph.argtypes = [vp, vp]
        L.bnm_plan_placement.argtypes = [vp, vp, vp]
        L.bnm_plan_window_tile.argtypes = [vp, vp, vp]
        L.bnm_philox_probe.argtypes = [i32, vp, i32, vp]
        L.bnm_calculate_params.argtypes = [i32, i32, i32, vp, dbl, dbl, dbl, dbl, vp, vp, vp, vp, vp]
        L.bnm_gof_noalloc.argtypes = [vp, i32, i32, i32, i32, i32, i32, i32, i32, dbl, vp, i32, vp, i32, vp, vp]
        L.bnm_run_simulations.argtypes = [vp] * 8 + [i32] * 6 + [vp, i32, vp, i32, i32, i32, i32, vp, i32, i32, i32,
                                                                 vp, vp, vp, vp]
        L.bnm_cmaes_params_default.argtypes = [C.POINTER(_CmaesParams)]
        L.bnm_cmaes_params_from_env.argtypes = [C.POINTER(_CmaesParams)]
        L.bnm_cmaes_create.argtypes = [C.POINTER(_CmaesParams), C.POINTER(vp)]
        L.bnm_cmaes_destroy.argtypes = [vp]
        L.bnm_cmaes_iteration.argtypes = [vp]
        L.bnm_cmaes_samples.argtypes = [vp, vp, vp, vp]
        L.bnm_cmaes_tell.argtypes = [vp, vp, vp]
        L.bnm_cmaes_best.argtypes = [vp, vp, vp]
        L.bnm_cmaes_set_samples.argtypes = [vp, vp]
        L.bnm_cmaes_state.argtypes = [vp, vp, vp, vp]
        L.bnm_cmaes_save.argtypes = [vp, C.c_char_p]
        L.bnm_cmaes_load.argtypes = [C.c_char_p, C.POINTER(vp)]
        L.bnm_cmaes_params_of.argtypes = [vp, C.POINTER(_CmaesParams)]
        _lib = L
    return _lib


def _check(rc: int):
    if rc != BNM_OK:
        raise BnmError(rc, lib().bnm_last_error().decode())


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _d(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


@dataclasses.dataclass
class Config:
    """Run configuration (the reference's CLI arguments + BNM_* settings)."""
    nodes: int = 100
    max_sims: int = 1
    time_steps: int = 60000
    bold_tr: int = 1000
    window_step: int = 2
    window_size: int = 10
    bold_remove_s: int = 30
    exc_interhem: bool = True
    do_fic: bool = True
    numerical_fic: bool = True
    max_fic_trials: int = 10
    i_sampling_start: int = 1000
    i_sampling_end: int = 10000
    init_delta: float = float(np.float32(0.02))
    use_fc_diff: bool = True
    fic_reject_failed: bool = False
    fic_penalty_scale: float = 2.0
    max_cost: float = 2.0
    calculate_fic_penalty: bool = True
    no_fcd: bool = False
    precision: int = PREC_F32
    noise_mode: int = NOISE_PHILOX
    noise_seed: int = 410
    device: int = 0
    gram: int = GRAM_AUTO  # split BF16 for PREC_F32, FP32 SIMT for the reference-order precisions

    @classmethod
    def from_env(cls, **overrides) -> "Config":
        c = _Config()
        lib().bnm_config_default(C.byref(c))
        lib().bnm_config_from_env(C.byref(c))
        kw = {f.name: getattr(c, f.name) for f in dataclasses.fields(cls)}
        kw.update(overrides)
        return cls(**kw)

    def _c(self) -> _Config:
        c = _Config()
        for f in dataclasses.fields(self):
            setattr(c, f.name, type(getattr(c, f.name))(getattr(self, f.name)))
        return c

    def sizes(self) -> dict:
        s = _Sizes()
        _check(lib().bnm_config_sizes(C.byref(self._c()), C.byref(s)))
        return {k: getattr(s, k) for k, _ in _Sizes._fields_}


class Plan:
    """Device-resident plan for one configuration (SC, targets, noise table,
    work space for ``cfg.max_sims`` particles)."""

    def __init__(self, cfg: Config, sc, emp_fc, emp_fcd=None, host_noise=None):
        self.cfg = cfg
        self.sizes = cfg.sizes()
        self._sc, self._efc = _d(sc), _d(emp_fc)
        self._efcd = _d(emp_fcd) if emp_fcd is not None else None
        nz = None
        if host_noise is not None:
            nz = np.ascontiguousarray(host_noise, dtype=np.float32)
        h = C.c_void_p()
        _check(lib().bnm_plan_create(C.byref(cfg._c()), _ptr(self._sc), _ptr(self._efc), len(self._efc),
                                     _ptr(self._efcd), 0 if self._efcd is None else len(self._efcd), _ptr(nz),
                                     0 if nz is None else nz.size, C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().bnm_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def run(self, G, wEE, wEI, wIE=None, outputs=("bold", "fc", "fcd", "ext_means", "w_ie")) -> dict:
        """One batch: returns cost, fic_penalty, fc_corr, fc_diff, fcd_ks,
        fic_failed, fic_ntrials, fic_unstable and the requested ``outputs``."""
        G = _d(np.atleast_1d(G))
        n, N = len(G), self.cfg.nodes
        wEE, wEI = _d(np.broadcast_to(wEE, (n, N))), _d(np.broadcast_to(wEI, (n, N)))
        wIE = None if wIE is None else _d(np.broadcast_to(wIE, (n, N)))
        s = self.sizes
        res = {k: np.zeros(n) for k in ("cost", "fic_penalty", "fc_corr", "fc_diff", "fcd_ks")}
        for k in ("fic_failed", "fic_ntrials", "fic_unstable"):
            res[k] = np.zeros(n, np.int32)
        shapes = {"w_ie": (n, N), "ext_means": (n, 6, N), "bold": (n, s["frames"], N), "fc": (n, s["n_pairs"]),
                  "fcd": (n, s["n_fcd"]), "fcd_left": (n, s["n_fcd"]), "fcd_right": (n, s["n_fcd"])}
        for k in outputs:
            res[k] = np.zeros(shapes[k])
        o = _BatchOut()
        for k, _ in _BatchOut._fields_:
            setattr(o, k, _ptr(res.get(k)))
        _check(lib().bnm_run(self._h, n, _ptr(G), _ptr(wEE), _ptr(wEI), _ptr(wIE), C.byref(o)))
        return res

    def check_fit_bold(self, bold, outputs=("fc", "fcd")) -> dict:
        """Goodness of fit of given BOLD (check_fit_bold, check_fit.cpp:138-217):
        ``bold`` [n, corr_len, N] kept frames.  Returns cost, fc_corr, fc_diff,
        fcd_ks and the requested ``outputs`` (fc, fcd)."""
        s = self.sizes
        bold = _d(np.asarray(bold))
        if bold.ndim != 3 or bold.shape[1:] != (s["corr_len"], self.cfg.nodes):
            raise ValueError(f"bold must be [n, {s['corr_len']}, {self.cfg.nodes}]")
        n = bold.shape[0]
        res = {k: np.zeros(n) for k in ("cost", "fic_penalty", "fc_corr", "fc_diff", "fcd_ks")}
        shapes = {"fc": (n, s["n_pairs"]), "fcd": (n, s["n_fcd"]), "fcd_left": (n, s["n_fcd"]),
                  "fcd_right": (n, s["n_fcd"])}
        for k in outputs:
            res[k] = np.zeros(shapes[k])
        o = _BatchOut()
        for k, _ in _BatchOut._fields_:
            setattr(o, k, _ptr(res.get(k)))
        _check(lib().bnm_check_fit_bold(self._h, n, _ptr(bold), C.byref(o)))
        return res

    def analytic_fic(self, G, wEE, wEI):
        G = _d(np.atleast_1d(G))
        n, N = len(G), self.cfg.nodes
        wEE, wEI = _d(np.broadcast_to(wEE, (n, N))), _d(np.broadcast_to(wEI, (n, N)))
        out, uns = np.zeros((n, N)), np.zeros(n, np.int32)
        _check(lib().bnm_analytic_fic(self._h, n, _ptr(G), _ptr(wEE), _ptr(wEI), _ptr(out), _ptr(uns)))
        return out, uns.astype(bool)

    def timings(self) -> dict:
        t = np.zeros(6)
        _check(lib().bnm_last_timings(self._h, _ptr(t)))
        return dict(zip(["fic", "integrate", "fc_window", "fcd_ks", "gof", "total"], t.tolist()))

    def gram_timing(self) -> dict:
        """Tensor-core Gram kernel times of the last call (ms) and the number of
        library kernels it launched."""
        t, k = np.zeros(2), C.c_int32()
        _check(lib().bnm_last_gram(self._h, _ptr(t), C.byref(k)))
        return dict(fc_gram_ms=float(t[0]), fcd_gram_ms=float(t[1]), launches=k.value)

    def window_tile(self) -> dict:
        """Window-FC tile the tuner picked (pairs per thread of a 256-thread CTA)."""
        t, k = C.c_int32(), C.c_int32()
        _check(lib().bnm_plan_window_tile(self._h, C.byref(t), C.byref(k)))
        return dict(pairs_per_thread=t.value, pairs_per_cta=256 * t.value, tried=k.value)

    def graph_launched(self) -> bool:
        """Whether the last run was one CUDA graph launch (bnm_plan_graph)."""
        g = C.c_int32()
        _check(lib().bnm_plan_graph(self._h, C.byref(g)))
        return bool(g.value)

    def placement(self) -> dict:
        """Particle placement state (bnm_plan_placement)."""
        e, l = C.c_int32(), C.c_int32()
        _check(lib().bnm_plan_placement(self._h, C.byref(e), C.byref(l)))
        return dict(enabled=bool(e.value), placed_last=bool(l.value))

    def integrator(self) -> dict:
        """FP32 integrator shape the autotuner picked for the last batch size."""
        o, t = np.zeros(5, np.int32), C.c_int32()
        _check(lib().bnm_plan_integrator(self._h, _ptr(o), C.byref(t)))
        kind = ["register", "cluster", "reference-order", "colsplit", "colsplit2"][int(o[0])]
        return dict(kind=kind, slots=int(o[1]), csize=int(o[2]), rpw=int(o[3]), kr=int(o[4]), tried=t.value)

    def noise(self, offset: int, n: int) -> np.ndarray:
        out = np.zeros(n, np.float32)
        _check(lib().bnm_plan_noise(self._h, offset, n, _ptr(out)))
        return out


class Group:
    """Several plans (subjects) run as one CUDA graph per generation
    (bnm_group_*): each plan on its own stream, one graph launch, one host
    synchronisation.  ``run`` takes per-plan (G, wEE, wEI) and returns per-plan
    dicts of cost, fic_penalty, fc_corr, fc_diff, fcd_ks, w_ie, fic_failed,
    fic_ntrials, fic_unstable."""

    def __init__(self, plans):
        self.plans = list(plans)
        arr = (C.c_void_p * len(self.plans))(*[p._h.value for p in self.plans])
        h = C.c_void_p()
        _check(lib().bnm_group_create(arr, len(self.plans), C.byref(h)))
        self._h = h

    def run(self, params) -> list:
        k = len(self.plans)
        if len(params) != k:
            raise ValueError(f"need {k} parameter sets")
        keep, res, outs = [], [], (_BatchOut * k)()
        n = (C.c_int32 * k)()
        Gp, Ep, Ip = (C.c_void_p * k)(), (C.c_void_p * k)(), (C.c_void_p * k)()
        for i, (p, (G, wEE, wEI)) in enumerate(zip(self.plans, params)):
            G = _d(np.atleast_1d(G))
            m, N = len(G), p.cfg.nodes
            wEE, wEI = _d(np.broadcast_to(wEE, (m, N))), _d(np.broadcast_to(wEI, (m, N)))
            keep += [G, wEE, wEI]
            n[i], Gp[i], Ep[i], Ip[i] = m, _ptr(G), _ptr(wEE), _ptr(wEI)
            r = {x: np.zeros(m) for x in ("cost", "fic_penalty", "fc_corr", "fc_diff", "fcd_ks")}
            r["w_ie"] = np.zeros((m, N))
            for x in ("fic_failed", "fic_ntrials", "fic_unstable"):
                r[x] = np.zeros(m, np.int32)
            for f, _ in _BatchOut._fields_:
                setattr(outs[i], f, _ptr(r.get(f)))
            res.append(r)
        _check(lib().bnm_group_run(self._h, n, Gp, Ep, Ip, outs))
        return res

    def last(self) -> dict:
        ms, g = C.c_double(), C.c_int32()
        _check(lib().bnm_group_last(self._h, C.byref(ms), C.byref(g)))
        return dict(ms=ms.value, graph=bool(g.value))

    def close(self):
        if self._h:
            lib().bnm_group_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def measure_fp32_peak(device: int = 0) -> float:
    """FP32 FMA-pipe throughput of the device in TFLOP/s (packed FMA probe)."""
    t = C.c_double()
    _check(lib().bnm_measure_fp32_peak(device, C.byref(t)))
    return t.value


def bw_math_probe(x, device: int = 0) -> np.ndarray:
    """[n, 4]: the Balloon-Windkessel step's e^x - 1 and ln(1 + x) next to
    CUDA's expm1f and log1pf (test support)."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.zeros((len(x), 4), np.float32)
    _check(lib().bnm_bw_math_probe(device, _ptr(x), len(x), _ptr(out)))
    return out


LOCAL_PARAMS = ("wee", "wie", "wei")  # bit order of het_mask (run_CMAES.cpp:252)


def calculate_params(nodes: int, G: float, wee: float, wie: float, wei: float, het=(), maps=None, scales=None):
    """bnm_calculate_params: one particle's G and per-node wEE / wEI / wIE.
    het: names of the regional parameters among LOCAL_PARAMS; maps [n_maps,
    nodes]; scales [3, n_maps] (map coefficients per local parameter, in
    LOCAL_PARAMS order)."""
    mask = sum(1 << LOCAL_PARAMS.index(h) for h in het)
    maps = _d(np.zeros((0, nodes)) if maps is None else maps).reshape(-1, nodes)
    scales = _d(np.zeros((3, max(len(maps), 1))) if scales is None else scales)
    g, ee, ei, ie = np.zeros(1), np.zeros(nodes), np.zeros(nodes), np.zeros(nodes)
    _check(lib().bnm_calculate_params(nodes, mask, len(maps), _ptr(maps) if len(maps) else None, float(G),
                                      float(wee), float(wie), float(wei), _ptr(scales), _ptr(g), _ptr(ee), _ptr(ei),
                                      _ptr(ie)))
    return g[0], ee, ei, ie


def philox_probe(counters_keys, device: int = 0) -> np.ndarray:
    """Device Philox4x32-10 block function: [n, 6] (counter[4], key[2]) ->
    [n, 4] output words (test support)."""
    x = np.ascontiguousarray(counters_keys, dtype=np.uint32).reshape(-1, 6)
    out = np.zeros((len(x), 4), np.uint32)
    _check(lib().bnm_philox_probe(device, _ptr(x), len(x), _ptr(out)))
    return out


def wait_probe(limit_ns: int, device: int = 0) -> dict:
    """bnm_wait_probe: a bounded device wait on an mbarrier that nothing
    arrives on, with a limit of ``limit_ns`` ns of wall time (test support).
    Returns the call's status code, the kernel's status word and the elapsed
    wait in ms; the expected code is BNM_ETIMEOUT."""
    st, ms = C.c_int32(0), C.c_double(0.0)
    rc = lib().bnm_wait_probe(device, int(limit_ns), C.byref(st), C.byref(ms))
    return {"code": rc, "status": st.value, "elapsed_ms": ms.value,
            "message": lib().bnm_last_error().decode() if rc else ""}


def gof_noalloc(d_bold: int, n: int, frames: int, nodes: int, n_vols_remove: int, window_size: int,
                window_step: int, emp_fc, emp_fcd, d_out: int, *, exc_interhem=True, use_fc_diff=True,
                max_cost=2.0, stream: int = 0) -> None:
    """bnm_gof_noalloc: goodness of fit of ``n`` BOLD series already on the
    device (``d_bold``: device address of float [n][frames][nodes]) into
    ``d_out`` (device address of double [5][n]: cost, fc_corr, fc_diff,
    fcd_ks, 0), using only the library's static device scratch array.
    Asynchronous on ``stream``."""
    efc = _d(emp_fc)
    efcd = np.sort(_d(emp_fcd))
    _check(lib().bnm_gof_noalloc(C.c_void_p(d_bold), n, frames, nodes, n_vols_remove, window_size, window_step,
                                 int(exc_interhem), int(use_fc_diff), float(max_cost), _ptr(efc), len(efc),
                                 _ptr(efcd), len(efcd), C.c_void_p(d_out), C.c_void_p(stream)))


def run_simulations(G_list, w_EE_list, w_EI_list, w_IE_list, SC, *, time_steps, BOLD_TR, window_size, window_step,
                    emp_FC_tril, emp_FCD_tril, max_fic_trials=10, do_fic=True, adjust_fic=True,
                    calculate_fic_penalty=True, sim_only=False, noise=None, rand_seed=410, w_IE_fic=None,
                    want_bold=False, want_ext=False):
    """Mirror of the reference's run_simulations (bnm.cu:594-617) through the
    one-shot C entry point.  Returns dict(corr, fic_penalties, w_IE_fic,
    FIC_failed, fic_n_trials[, BOLD_ex, ext_means])."""
    G = _d(np.atleast_1d(G_list))
    n, N = len(G), SC.shape[0]
    wEE, wEI = _d(np.broadcast_to(w_EE_list, (n, N))), _d(np.broadcast_to(w_EI_list, (n, N)))
    wIE = _d(np.broadcast_to(w_IE_list, (n, N)))
    corr, pen = np.zeros(n), np.zeros(n)
    wfic = None if w_IE_fic is None else _d(np.broadcast_to(w_IE_fic, (n, N))).copy()
    failed, trials = np.zeros(n, np.int32), np.zeros(n, np.int32)
    frames = time_steps // BOLD_TR + 1
    bold = np.zeros((n, frames, N)) if want_bold else None
    ext = np.zeros((n, 6, N)) if want_ext else None
    efc, efcd = _d(emp_FC_tril), _d(emp_FCD_tril)
    nz = None if noise is None else np.ascontiguousarray(noise, dtype=np.float32)
    _check(lib().bnm_run_simulations(_ptr(corr), _ptr(pen), _ptr(G), _ptr(wEE), _ptr(wEI), _ptr(wIE), _ptr(wfic),
                                     _ptr(_d(SC)), N, int(calculate_fic_penalty), time_steps, BOLD_TR,
                                     max_fic_trials, int(sim_only), _ptr(efc), len(efc), _ptr(efcd), len(efcd),
                                     window_size, window_step, n, _ptr(nz), rand_seed, int(do_fic), int(adjust_fic),
                                     _ptr(failed), _ptr(trials), _ptr(bold), _ptr(ext)))
    out = dict(corr=corr, fic_penalties=pen, w_IE_fic=wfic, FIC_failed=failed, fic_n_trials=trials)
    if want_bold:
        out["BOLD_ex"] = bold
    if want_ext:
        out["ext_means"] = ext
    return out


class CMAES:
    """Host CMA-ES with the reference's CMAES_Points semantics."""

    def __init__(self, lambda_: int, dimension: int, seed_mw: int, it_max: int, from_env: bool = True, **kw):
        p = _CmaesParams()
        lib().bnm_cmaes_params_default(C.byref(p))
        if from_env:
            lib().bnm_cmaes_params_from_env(C.byref(p))
        p.lambda_, p.dimension, p.seed_mw, p.it_max = lambda_, dimension, seed_mw, it_max
        for k, v in kw.items():
            setattr(p, k, v)
        h = C.c_void_p()
        if lib().bnm_cmaes_create(C.byref(p), C.byref(h)) != 0:
            raise BnmError(BNM_EINVAL, "bad CMA-ES parameters")
        self._h, self.lam, self.dim, self.it_max = h, lambda_, dimension, it_max

    def __del__(self):
        if getattr(self, "_h", None):
            lib().bnm_cmaes_destroy(self._h)
            self._h = None

    @property
    def iteration(self) -> int:
        return lib().bnm_cmaes_iteration(self._h)

    def samples(self):
        f, r, p = (np.zeros((self.dim, self.lam)) for _ in range(3))
        lib().bnm_cmaes_samples(self._h, _ptr(f), _ptr(r), _ptr(p))
        return f, r, p

    def set_samples(self, raw):
        """Replace this generation's raw samples ([dim][lambda]) before tell()."""
        raw = np.ascontiguousarray(raw, dtype=np.float64).reshape(self.dim, self.lam)
        if lib().bnm_cmaes_set_samples(self._h, _ptr(raw)) != 0:
            raise BnmError(BNM_EINVAL, "bad samples")

    def tell(self, cost):
        pen = np.zeros(self.lam)
        it = lib().bnm_cmaes_tell(self._h, _ptr(_d(cost)), _ptr(pen))
        return it, pen

    def best(self):
        x, v = np.zeros(self.dim), C.c_double()
        lib().bnm_cmaes_best(self._h, _ptr(x), C.byref(v))
        return x, v.value

    def state(self):
        m, s, Cm = np.zeros(self.dim), C.c_double(), np.zeros((self.dim, self.dim))
        lib().bnm_cmaes_state(self._h, _ptr(m), C.byref(s), _ptr(Cm))
        return m, s.value, Cm

    def save(self, path: str):
        """Checkpoint the whole optimiser state to path (bnm_cmaes_save)."""
        rc = lib().bnm_cmaes_save(self._h, os.fsencode(path))
        if rc != 0:
            raise BnmError(BNM_EINVAL, f"cannot write CMA-ES checkpoint {path} ({rc})")

    @classmethod
    def load(cls, path: str) -> "CMAES":
        """An optimiser resumed from a checkpoint (bnm_cmaes_load)."""
        h = C.c_void_p()
        rc = lib().bnm_cmaes_load(os.fsencode(path), C.byref(h))
        if rc != 0:
            raise BnmError(BNM_EINVAL, f"cannot read CMA-ES checkpoint {path} ({rc})")
        self = cls.__new__(cls)
        self._h = h
        p = _CmaesParams()
        lib().bnm_cmaes_params_of(h, C.byref(p))
        self.lam, self.dim, self.it_max = p.lambda_, p.dimension, p.it_max
        return self
