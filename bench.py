#!/usr/bin/env python
"""Benchmark of the simulate-and-fit hot path: one CMA-ES generation.

Workload (one step): 256 particles sharing one synthetic 100-node connectome
(30 % density, log-normal weights, max row sum 1, seed 0), each simulated for
450 s of model time (dt 0.1 ms, 4.5 M Euler-Maruyama substeps) with analytic
+ numerical FIC (up to 10 restarts), Balloon-Windkessel BOLD at TR 0.72 s
(626 frames, 41 removed), FC (2450 pairs), sliding-window FC (window 44 TRs,
step 1: 541 windows), FCD (146,070 entries), the KS distance to a target FCD
and the goodness of fit.  Parameters: G uniform on [0.5, 4], wEE and wEI
uniform on [0.05, 0.75].  Targets: the model's own FC/FCD at G=2, wEE=0.3,
wEI=0.2 (synthetic, seeded).  Noise: device Philox table, seed 410.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints one JSON line.  ``value`` is sims/s from the device-side stage timers
(CUDA events on the plan's stream) with every input resident in HBM; ``e2e``
is sims/s through the public C-ABI call (bnm_run) with host buffers: parameter
upload and result download are inside the timed region.  Under torchrun each
rank runs its own generation (weak scaling) and the costs are all-gathered,
as a host CMA-ES needs them; times are the max over ranks.

``--impl reference`` times the reference's own OpenMP CPU path (bnm.cpp,
compiled from its sources, oracle/_ref) on every host core.  Its value is a
measurement made once per invocation: one particle per core, each simulated
for the full 450 s with FIC and analysed to its cost, timed per simulation
(sims/s = cores / mean seconds per simulation).  Each timed step is a bounded
sample (one particle per core for 12 s of model time, enough for the FIC
window and every restart) extrapolated to full simulations by the substeps
executed, with the FIC restart counts of the full run and the reference's
measured FC/FCD/KS time; that extrapolation is reported beside the measured
value.  The GPU arm's cpu_baseline carries the same two figures.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_NODES, N_SIMS, T_MS, TR, WS, STEP, REMOVE_S = 100, 256, 450_000, 720, 44, 1, 30
DEFAULT_SIMS, DEFAULT_T_MS = N_SIMS, T_MS
SAMPLE_MS = 12_000
WORKLOAD = "cmaes-generation-N100-450s-x256"


def workload_inputs(world: int = 1, seed: int = 1):
    """SC and the whole population: N_SIMS particles per rank (weak scaling);
    rank r simulates particles [r N_SIMS, (r+1) N_SIMS) (bnm_cuda_b200.shard).
    The particles are a uniform draw on the parameter bounds (seed 1: the
    first timed generation and the CPU reference's particles)."""
    from bnm_cuda_b200 import synth

    sc = synth.make_sc(N_NODES, 0.3, 0)
    G, wEE, wEI = synth.uniform_params(N_SIMS * world, N_NODES, seed)
    return sc, G, wEE, wEI


def generation_seeds(warmup: int, steps: int):
    """Particle seeds of the warm-up and timed generations: every generation
    draws new particles (as CMA-ES does), so the plan's placement history never
    holds the particles it places."""
    return [1001 + w for w in range(warmup)], [1 + k for k in range(steps)]


def make_targets(sc):
    """The model's own FC/FCD at G=2, wEE=0.3, wEI=0.2 (device, FP32, Philox seed 1)."""
    import bnm_cuda_b200 as B

    cfg = B.Config(nodes=N_NODES, max_sims=1, time_steps=T_MS, bold_tr=TR, window_size=WS, window_step=STEP,
                   bold_remove_s=REMOVE_S, noise_seed=1)
    s = cfg.sizes()
    with B.Plan(cfg, sc, np.zeros(s["n_pairs"]), np.zeros(s["n_fcd"])) as p:
        r = p.run(2.0, 0.3, 0.2, outputs=("fc", "fcd"))
    return r["fc"][0], r["fcd"][0]


class ClockSampler:
    """nvidia-smi samples (200 ms) of SM clock and throttle reasons."""

    def __init__(self, device: int):
        self.device, self.proc, self.path = device, None, None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait(timeout=10)

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    mx = max(mx, float(f[2]))
                except ValueError:
                    continue
                for n, v in zip(names, f[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
        except OSError:
            pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ CPU side
class _QuietStdout:
    """Silence C-level stdout (the reference prints one line per particle)."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        devnull = os.open(os.devnull, os.O_WRONLY)
        os.dup2(devnull, 1)
        os.close(devnull)

    def __exit__(self, *a):
        os.dup2(self.saved, 1)
        os.close(self.saved)


_FULL = {}


def _targets_for_cpu():
    """Seeded stand-in targets of the workload's sizes (2450 FC pairs, 146,070
    FCD entries) for the reference's CPU runs: the GOF costs the same time for
    any values, and the GPU-made targets are not available to the CPU arm."""
    rng = np.random.default_rng(2)
    return rng.uniform(-0.2, 0.8, 2450), rng.uniform(-0.3, 1.0, 146_070)


def cpu_reference_full(n_threads: int, fp32: bool = False):
    """One full-length measurement of the reference's CPU path: the first
    n_threads particles of the workload, one per core, each simulated for the
    whole 450 s with FIC and analysed (FC, window FC, FCD, KS, cost) by the
    reference's own bnm() (the body of run_simulations' OpenMP loop,
    bnm.cpp:441-465), timed per particle.  The FIC trial counts come from the
    reference's own output files.  Cached per process.  Returns a dict with
    the measured sims/s (= cores / mean seconds per simulation: every core
    busy with whole simulations, as in a 256-particle generation) and the
    per-particle seconds and trial counts."""
    key = (n_threads, fp32)
    if key in _FULL:
        return _FULL[key]
    os.environ.setdefault("OMP_NUM_THREADS", str(n_threads))
    from oracle import ref

    if not ref.ref_available(fp32):
        return None
    sc, G, wEE, wEI = workload_inputs(1)
    idx = np.arange(n_threads) % N_SIMS
    emp_fc, emp_fcd = _targets_for_cpu()
    with tempfile.TemporaryDirectory() as d, _QuietStdout():
        t0 = time.perf_counter()
        r = ref.ref_run_particles_timed(sc, G[idx], wEE[idx], wEI[idx], np.zeros((len(idx), N_NODES)),
                                        time_steps=T_MS, bold_tr=TR, rand_seed=410, max_fic_trials=10,
                                        emp_fc=emp_fc, emp_fcd=emp_fcd, window_step=STEP, window_size=WS,
                                        out_dir=d, fp32=fp32)
        wall = time.perf_counter() - t0
    sec = r["seconds"]
    _FULL[key] = dict(value=n_threads / float(sec.mean()), wall_s=wall, seconds=sec, trials=r["trials"],
                      sample=f"{len(idx)} particles x {T_MS} ms (the workload's first {len(idx)}, 1 per core, FIC "
                             f"on, full FC/FCD/KS/cost), measured end to end; value = cores / mean seconds per "
                             f"simulation ({sec.mean():.1f} s; slowest {sec.max():.1f} s)")
    return _FULL[key]


def cpu_reference_sample(n_threads: int, sample_ms: int = SAMPLE_MS, fp32: bool = False, trials=None):
    """One bounded sample of the reference's CPU run_simulations
    (bnm.cpp:431-466): the same particles as cpu_reference_full, one per core,
    for sample_ms of model time (enough for the FIC sampling window and every
    FIC restart), extrapolated to full simulations by the substeps executed
    (10 (T+1) + 100,000 per FIC restart, with the restart counts the
    reference's own full-length run reported), plus the reference's measured
    FC / FCD / KS time for one full-size BOLD series.  fp32 times the
    reference's -DUSE_FLOATS build.  Returns (sims_per_s, detail)."""
    os.environ.setdefault("OMP_NUM_THREADS", str(n_threads))
    from oracle import ref

    if not ref.ref_available(fp32):
        return None
    sc, G, wEE, wEI = workload_inputs(1)
    idx = np.arange(n_threads) % N_SIMS
    n = len(idx)
    zeros = np.zeros((n, N_NODES))
    fic = sample_ms >= 10_000
    with _QuietStdout():
        t0 = time.perf_counter()
        ref.ref_run_simulations(sc, G[idx], wEE[idx], wEI[idx], zeros if fic else zeros + 1.0, time_steps=sample_ms,
                                bold_tr=1000, rand_seed=410, max_fic_trials=10, emp_fc=np.zeros(2450),
                                emp_fcd=np.zeros(10), window_step=1, window_size=2, sim_only=True, fp32=fp32)
        t_sample = time.perf_counter() - t0
    if not fic or trials is None:
        return None
    tr = np.asarray(trials, np.float64)
    s_sample = 10 * (sample_ms + 1) + 100_000 * tr
    s_full = 10 * (T_MS + 1) + 100_000 * tr
    rate = s_sample.max() / t_sample  # substeps per second per core (threads run in parallel)
    # the reference's FC / FCD / KS on one full-size BOLD series
    bold = np.random.default_rng(0).standard_normal((626 - 41, N_NODES)) * 0.01
    emp_fc, emp_fcd = _targets_for_cpu()
    t1 = time.perf_counter()
    with _QuietStdout():
        ref.ref_check_fit_bold(bold, STEP, WS, emp_fc, emp_fcd, fp32=fp32)
    t_gof = time.perf_counter() - t1
    per_sim = s_full.mean() / rate + t_gof
    sims_per_s = n_threads / per_sim
    return sims_per_s, {"sample": f"{n} particles x {sample_ms} ms model time (1 per core, FIC on), scaled by "
                                  f"substeps to {T_MS} ms with the reference's own FIC restart counts + one full "
                                  f"FC/FCD/KS ({t_gof:.2f} s)",
                        "sample_s": t_sample + t_gof, "per_sim_s": per_sim}


TRAFFIC_FILE = os.path.join(ROOT, "profiles", "integrate_fast_kernel_N100_70s_x256_traffic.txt")


def integrator_traffic() -> dict:
    """roofline.traffic of the integrator: DRAM bytes (read + write) of one
    launch from the committed ncu capture (a 70 s, 256-particle case of the
    same kernel and noise source), scaled to this run's model time; null when
    the summary is missing."""
    try:
        kv = dict(line.split(None, 1) for line in open(TRAFFIC_FILE) if line.strip() and not line.startswith("#"))
        b, ms = float(kv["dram_bytes_per_launch"]), float(kv["model_ms"])
    except (OSError, KeyError, ValueError):
        return {"traffic": None, "traffic_source": "no committed capture"}
    return {"traffic": b * (T_MS + 1) / (ms + 1),
            "traffic_source": f"ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch at {int(ms)} ms model "
                              f"time ({b / 1e6:.1f} MB), scaled to {T_MS} ms ({os.path.relpath(TRAFFIC_FILE, ROOT)})"}


def workload_config(world: int = 1) -> dict:
    """The workload as both arms report it (same keys and values)."""
    return {"workload": WORKLOAD, "nodes": N_NODES, "particles_per_gpu": N_SIMS, "model_time_ms": T_MS,
            "tr_ms": TR, "window": WS, "step": STEP, "fic": "analytic + numerical, up to 10 restarts",
            "particles": "uniform on the parameter bounds, a fresh draw every generation (timed: seeds 1, 2, ...; "
                         "warm-up: 1001, ...)",
            "l2": "inputs larger than L2 (3.6 GB noise stream, 1.4 GB window FC per generation)",
            "parallelism": f"particles sharded over {world} GPU(s)"}


def run_reference(args):
    """The reference's OpenMP CPU path on every host core.  Timed steps are
    bounded samples (cpu_reference_sample); the value is the full-length
    measurement (cpu_reference_full), made once per invocation, with the
    samples' extrapolated figure beside it."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", str(args.gpus)))
    if rank != 0:
        return 0
    cores = len(os.sched_getaffinity(0))
    from oracle import ref

    if not ref.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref reference build missing"}))
        return 0
    full = cpu_reference_full(cores)
    for i in range(args.warmup):  # short, FIC-free warm-up samples
        cpu_reference_sample(cores, sample_ms=2_000)
    vals, secs = [], []
    for i in range(args.steps):
        t0 = time.perf_counter()
        r = cpu_reference_sample(cores, trials=full["trials"])
        secs.append(time.perf_counter() - t0)
        vals.append(r[0])
    modelled = float(np.mean(vals))
    v = full["value"]
    print(json.dumps({
        "impl": "reference", "metric": "sims/s", "value": v, "unit": "sims/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * float(np.mean(secs)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(world),
        "cpu_baseline": {"value": v, "unit": "sims/s", "cores": cores, "kind": "reference", "sample": full["sample"],
                         "measured_full": _full_summary(full),
                         "modelled": {"value": modelled, "sample": r[1]["sample"],
                                      "measured_over_modelled": v / modelled}},
        "step_note": "each timed step is one bounded sample (ms_per_step is its wall time); value is the "
                     "full-length measurement made once before them",
        "e2e": {"value": v, "unit": "sims/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))
    return 0


def _full_summary(full):
    return {"value": full["value"], "wall_s": full["wall_s"], "mean_s_per_sim": float(full["seconds"].mean()),
            "max_s_per_sim": float(full["seconds"].max()), "fic_restarts": [int(t) for t in full["trials"]],
            "sample": full["sample"]}


# ------------------------------------------------------------------ GPU side
def run_b200(args):
    import bnm_cuda_b200 as B

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    from bnm_cuda_b200 import shard

    warm_seeds, step_seeds = generation_seeds(args.warmup, args.steps)
    sc = workload_inputs(world)[0]
    gens = {k: workload_inputs(world, k)[1:] for k in warm_seeds + step_seeds}  # host arrays, made before timing
    a, b = shard.shard_bounds(N_SIMS * world, world, rank)
    emp_fc, emp_fcd = make_targets(sc)
    gram = {"f32": B.GRAM_F32, "bf16": B.GRAM_BF16, "bf16x3": B.GRAM_BF16_SPLIT}[args.gram]
    cfg = B.Config(nodes=N_NODES, max_sims=N_SIMS, time_steps=T_MS, bold_tr=TR, window_size=WS, window_step=STEP,
                   bold_remove_s=REMOVE_S, noise_seed=410, device=local, gram=gram)
    plan = B.Plan(cfg, sc, emp_fc, emp_fcd)
    outputs = ("w_ie",)  # the reference returns corr, fic_penalties, w_IE_fic, FIC_failed, fic_n_trials
    for k in warm_seeds:
        G_all, wEE_all, wEI_all = gens[k]
        plan.run(G_all[a:b], wEE_all[a:b], wEI_all[a:b], outputs=outputs)

    def barrier():
        if dist:
            import torch
            torch.cuda.synchronize()
            dist.barrier()

    barrier()
    dev_ms, integ_ms, wall, flops, launches, placed = [], [], [], [], 0, 0
    with ClockSampler(local) as clk:
        for k in step_seeds:
            G_all, wEE_all, wEI_all = gens[k]
            t0 = time.perf_counter()
            if dist:  # this rank's shard, then every particle's fit terms on every rank (NCCL)
                r = shard.run_sharded(lambda g, e, i: plan.run(g, e, i, outputs=outputs), G_all, wEE_all, wEI_all)
                torch.cuda.synchronize()
            else:
                r = plan.run(G_all, wEE_all, wEI_all, outputs=outputs)
            wall.append(time.perf_counter() - t0)
            t = plan.timings()
            launches += plan.gram_timing()["launches"]
            placed += plan.placement()["placed_last"]
            dev_ms.append(t["total"])
            integ_ms.append(t["integrate"])
            subs = 10 * (T_MS + 1) + 100_000 * np.asarray(r["fic_ntrials"], np.float64)[a:b] if dist else \
                10 * (T_MS + 1) + 100_000 * r["fic_ntrials"].astype(np.float64)
            flops.append(2.0 * N_NODES * N_NODES * subs.sum())
    barrier()
    dev_total, wall_total = float(np.sum(dev_ms)) / 1e3, float(np.sum(wall))
    if dist:
        import torch
        t = torch.tensor([dev_total, wall_total], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dev_total, wall_total = t.tolist()
    value = world * N_SIMS * args.steps / dev_total
    e2e = world * N_SIMS * args.steps / wall_total
    result = None
    if rank == 0:
        peak = B.measure_fp32_peak(local)
        achieved = float(np.mean(np.array(flops) / (np.array(integ_ms) * 1e-3))) / 1e12
        cores = len(os.sched_getaffinity(0))
        full = cpu_reference_full(cores) if (world == 1 and not args.no_cpu) else None
        cpu = cpu_reference_sample(cores, trials=full["trials"]) if full else None
        cpu32 = cpu_reference_sample(cores, fp32=True, trials=full["trials"]) if full else None
        n, N = N_SIMS, N_NODES
        result = {
            "metric": "sims/s", "value": value, "unit": "sims/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * dev_total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(world),
            "impl_config": {"precision": "f32 integration, f64 FIC/centring", "gram": args.gram,
                            "integrator": plan.integrator(), "window_tile": plan.window_tile(),
                            "noise": "philox table", "graph_launched": plan.graph_launched(),
                            "placement": {**plan.placement(), "placed_steps": placed}},
            "e2e": {"value": e2e, "unit": "sims/s", "h2d_bytes_per_step": 8 * (n + 2 * n * N),
                    "d2h_bytes_per_step": 8 * n * 5 + 4 * n * 3 + 8 * n * N},
            "gpu_launches": launches,
            "roofline": {"bound": "fp32", "kernel": "integrate_fast_kernel", "achieved": achieved,
                         "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                         **integrator_traffic(),
                         "peak_source": "measured on this GPU by bnm_measure_fp32_peak (packed FP32 FMA chains)",
                         "work": "2*N^2 FLOP per substep per particle (coupling FMAs only), FIC restarts included"},
            "stage_ms": {k: float(v) for k, v in plan.timings().items()},
            "clocks": clk.summary(),
        }
        if cpu is not None:
            result["cpu_baseline"] = {"value": cpu[0], "unit": "sims/s", "cores": cores,
                                      "kind": "reference", "sample": cpu[1]["sample"],
                                      "measured_full": _full_summary(full),
                                      "modelled_over_measured": cpu[0] / full["value"]}
        if cpu32 is not None:  # the reference's float build (-DUSE_FLOATS), same sample
            result["cpu_baseline_f32"] = {"value": cpu32[0], "unit": "sims/s", "cores": cores,
                                          "kind": "reference", "sample": cpu32[1]["sample"]}
    plan.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if result is not None:
        print(json.dumps(result))
    return 0


def run_surrogate(args):
    """Surrogate-screened vs plain CMA-ES (second metric): N=100, 300 s at TR 1 s,
    window 44 step 1, FIC on; surrogate trained once on --train-sims uniform
    simulations; CMA-ES lambda=64 for --generations generations, screened
    runs sample 8x lambda and simulate the best lambda by predicted cost.

    Over --surrogate-seeds CMA-ES seeds (each screened run starts from the
    same trained network), like for like: the target of a seed is the plain
    run's final best plus 0.01, and each run's time-to-target is its wall time
    until its best is at or below that target (for the plain run, its own
    time to come within 0.01 of its final best, not its whole run).  Reported
    per seed (also against the better of the two final bests) and as the
    median ratio screened / plain, without and with the surrogate's one-off
    cost (training simulations + fit) added to the screened run; a screened
    run that never reaches the target counts as +inf."""
    import bnm_cuda_b200 as B
    from bnm_cuda_b200 import surrogate as S, synth

    sc = synth.make_sc(N_NODES, 0.3, 0)
    cfg = B.Config(nodes=N_NODES, max_sims=2048, time_steps=300_000, bold_tr=1000, window_size=WS, window_step=1,
                   bold_remove_s=REMOVE_S, noise_seed=410)
    s = cfg.sizes()
    tcfg = B.Config(**{**cfg.__dict__, "max_sims": 1, "noise_seed": 1})
    with B.Plan(tcfg, sc, np.zeros(s["n_pairs"]), np.zeros(s["n_fcd"])) as tp:
        tr = tp.run(2.0, 0.3, 0.2, outputs=("fc", "fcd"))
    bounds, spec = S.Bounds(), S.spectral_summary(sc)

    def to_target(run, target):
        for b, w in zip(run["best_hist"], run["wall_hist"]):
            if b <= target:
                return w
        return None

    seeds = []
    with B.Plan(cfg, sc, tr["fc"][0], tr["fcd"][0]) as plan:
        mlp, info = S.train_surrogate(plan, bounds, spec, n_train=args.train_sims, seed=0, epochs=args.epochs)
        trained = mlp.get_params()
        t_surrogate = info["sim_s"] + info["fit_s"]
        for seed in range(1, args.surrogate_seeds + 1):
            plain = S.run_cmaes(plan, bounds, 64, args.generations, seed=seed)
            mlp.set_params(trained)
            screen = S.run_cmaes(plan, bounds, 64, args.generations, seed=seed, mlp=mlp, spec=spec, oversample=8,
                                 holdout_spearman=info["holdout_spearman"])
            # the target: within 0.01 of plain CMA-ES's final best
            target = plain["best"] + 0.01
            tp_, ts_ = to_target(plain, target), to_target(screen, target)
            # and the better of the two final bests + 0.01: a run that never gets there loses outright
            better = min(plain["best"], screen["best"]) + 0.01
            bp, bs = to_target(plain, better), to_target(screen, better)
            seeds.append({"seed": seed, "plain_best": plain["best"], "screened_best": screen["best"],
                          "target": target, "plain_time_s": tp_, "screened_time_s": ts_,
                          "ratio": ts_ / tp_ if ts_ is not None else None,
                          "ratio_with_training": (ts_ + t_surrogate) / tp_ if ts_ is not None else None,
                          "better_target": better, "plain_time_to_better_s": bp, "screened_time_to_better_s": bs,
                          "plain_wall_s": plain["wall_hist"][-1], "screened_wall_s": screen["wall_hist"][-1],
                          "screened_generations": screen["screened_generations"],
                          "plain_hist": [round(b, 4) for b in plain["best_hist"]],
                          "screened_hist": [round(b, 4) for b in screen["best_hist"]],
                          "plain_walls": [round(w, 3) for w in plain["wall_hist"]],
                          "screened_walls": [round(w, 3) for w in screen["wall_hist"]]})
    # a seed whose screened run never comes within 0.01 of plain's best counts as a loss (ratio +inf)
    r_all = [r["ratio"] if r["ratio"] is not None else float("inf") for r in seeds]
    r_all_t = [r["ratio_with_training"] if r["ratio_with_training"] is not None else float("inf") for r in seeds]
    med, med_t = float(np.median(r_all)), float(np.median(r_all_t))
    print(json.dumps({
        "metric": "CMA-ES time to within 0.01 of plain's final best, surrogate-screened / plain (median over seeds)",
        "value": med if np.isfinite(med) else None, "unit": "fraction of plain time-to-target",
        "value_with_training": med_t if np.isfinite(med_t) else None,
        "screened_reached_target": sum(r["ratio"] is not None for r in seeds), "seeds_run": len(seeds),
        "higher_is_better": False, "data": "synthetic",
        "config": {"workload": "cmaes-surrogate-N100-300s-lambda64x8", "train_sims": args.train_sims,
                   "generations": args.generations, "seeds": args.surrogate_seeds,
                   "target": "plain CMA-ES final best + 0.01, per seed (time of the first generation at or "
                             "below it; a screened run that never gets there counts as +inf)"},
        "seeds": seeds, "surrogate_one_off_s": t_surrogate,
        "surrogate": {k: v for k, v in info.items() if k != "losses"},
    }))
    return 0


def fp64_fc_fcd(bold_kept, ws, step, exc):
    """FP64 restatement of the reference's FC, window FC and FCD (check_fit.cpp:19-134)
    for one BOLD series of kept frames [T, N]: pairs i > j row-major (optionally
    without inter-hemispheric pairs), windows centred ws/2 .. T-1-ws/2 by step."""
    T, N = bold_kept.shape
    i, j = np.tril_indices(N, -1)
    if exc:
        keep = ~((i < N // 2) ^ (j < N // 2))
        i, j = i[keep], j[keep]
    y = bold_kept - bold_kept.mean(0)
    ss = np.sqrt((y * y).sum(0))
    fc = (y.T @ y)[i, j] / (ss[i] * ss[j])
    h = ws // 2
    centres = range(h, T - h, step)
    wfc = np.empty((len(centres), len(i)))
    for k, c in enumerate(centres):
        yw = bold_kept[c - h:c + h + 1]
        yw = yw - yw.mean(0)
        sw = np.sqrt((yw * yw).sum(0))
        wfc[k] = (yw.T @ yw)[i, j] / (sw[i] * sw[j])
    z = wfc - wfc.mean(1, keepdims=True)
    z /= np.sqrt((z * z).sum(1, keepdims=True))
    a, b = np.tril_indices(len(centres), -1)
    return fc, (z @ z.T)[a, b]


def ks_2samp(x, y):
    """Two-sample Kolmogorov-Smirnov distance sup |F_x - F_y|."""
    x, y = np.sort(x), np.sort(y)
    v = np.concatenate([x, y])
    return float(np.max(np.abs(np.searchsorted(x, v, "right") / len(x) - np.searchsorted(y, v, "right") / len(y))))


def run_precision(args):
    """Precision stress on FC / FCD: 64 particles, N = 400 (10 % density SC,
    seed 0), 600 s at TR 0.5 s (1201 frames, none removed), window 44 step 1
    (1157 windows), all 79,800 pairs.  The batch is integrated once (FP32);
    its BOLD is then analysed with each Gram arithmetic through
    bnm_check_fit_bold: FP32 SIMT FCD + FP64 co-moment FC, tcgen05 BF16, and
    tcgen05 split BF16 (hi + lo).  Errors are against an FP64 restatement of
    the reference formulas on --check-sims particles: max |error| over FC
    entries, FCD entries, and of the KS distance to the target FCD."""
    import bnm_cuda_b200 as B
    from bnm_cuda_b200 import synth

    # --particles / --model-ms / --nodes (profiling knobs) replace the 64 particles, 600 s and 400 nodes
    n = args.particles if args.particles != DEFAULT_SIMS else 64
    T = args.model_ms if args.model_ms != DEFAULT_T_MS else 600_000
    N, TRp, WSp, STEPp = args.nodes, 500, 44, 1
    sc = synth.make_sc(N, 0.1, 0)
    G, wEE, wEI = synth.uniform_params(n, N, 1)
    cfg = B.Config(nodes=N, max_sims=n, time_steps=T, bold_tr=TRp, window_size=WSp, window_step=STEPp,
                   bold_remove_s=0, exc_interhem=False, noise_seed=410, gram=B.GRAM_F32)
    s = cfg.sizes()
    tcfg = B.Config(**{**cfg.__dict__, "max_sims": 1, "noise_seed": 1})
    with B.Plan(tcfg, sc, np.zeros(s["n_pairs"]), np.zeros(s["n_fcd"])) as tp:
        tr = tp.run(2.0, 0.3, 0.2, outputs=("fc", "fcd"))
    emp_fc, emp_fcd = tr["fc"][0], tr["fcd"][0]
    out = {}
    with ClockSampler(0) as clk:
        with B.Plan(cfg, sc, emp_fc, emp_fcd) as p:
            t0 = time.perf_counter()
            r = p.run(G, wEE, wEI, outputs=("bold", "fc", "fcd"))
            wall = time.perf_counter() - t0
            tm = p.timings()
            integ = p.integrator()
        kept = r["bold"][:, s["n_vols_remove"]:]
        out["f32"] = dict(fc=r["fc"], fcd=r["fcd"], ks=r["fcd_ks"], stage_ms=tm, gram=None)
        for name, gram in (("bf16", B.GRAM_BF16), ("bf16x3", B.GRAM_BF16_SPLIT)):
            gcfg = B.Config(**{**cfg.__dict__, "gram": gram})
            with B.Plan(gcfg, sc, emp_fc, emp_fcd) as q:
                for _ in range(2):  # second call timed (first loads the kernels)
                    f = q.check_fit_bold(kept)
                out[name] = dict(fc=f["fc"], fcd=f["fcd"], ks=f["fcd_ks"], stage_ms=q.timings(), gram=q.gram_timing())
    k = min(args.check_sims, n)
    ref = [fp64_fc_fcd(kept[i], WSp, STEPp, False) for i in range(k)]
    ks64 = [ks_2samp(emp_fcd, ref[i][1]) for i in range(k)]
    W, P = s["n_windows"], s["n_pairs"]
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {"bf16_tflops": 1590.0}
    rb = (W + 127) // 128
    kpad = ((P + 63) // 64) * 64
    table = {}
    for name, o in out.items():
        e = dict(fc_max_abs_err=max(float(np.abs(o["fc"][i] - ref[i][0]).max()) for i in range(k)),
                 fcd_max_abs_err=max(float(np.abs(o["fcd"][i] - ref[i][1]).max()) for i in range(k)),
                 fcd_mean_abs_err=float(np.mean([np.abs(o["fcd"][i] - ref[i][1]).mean() for i in range(k)])),
                 ks_max_abs_err=max(abs(float(o["ks"][i]) - ks64[i]) for i in range(k)),
                 fcd_stage_ms=o["stage_ms"]["fcd_ks"])
        if o["gram"]:
            prods = 3 if name == "bf16x3" else 1
            mma_flop = n * rb * (rb + 1) / 2 * 128 * 128 * kpad * 2 * prods
            ms = o["gram"]["fcd_gram_ms"]
            e.update(fcd_gram_ms=ms, tensor_tflops=mma_flop / (ms * 1e-3) / 1e12,
                     tensor_frac=mma_flop / (ms * 1e-3) / 1e12 / peaks["bf16_tflops"],
                     lower_triangle_tflops=n * W * (W - 1) * P * prods / (ms * 1e-3) / 1e12)
        table[name] = e
    print(json.dumps({
        "metric": "sims/s", "value": n / (tm["total"] / 1e3), "unit": "sims/s", "n_gpus": 1, "steps": 1,
        "higher_is_better": True, "data": "synthetic", "dtype": "f32 integration; FC/FCD Grams f32 / bf16 / bf16x3",
        "config": {"workload": f"precision-stress-N{N}-{T // 1000}s-x{n}", "nodes": N, "particles": n, "model_time_ms": T,
                   "tr_ms": TRp, "window": WSp, "step": STEPp, "windows": W, "pairs": P, "fcd_entries": s["n_fcd"],
                   "sc_density": 0.1, "integrator": integ, "checked_particles": k},
        "wall_s": wall, "stage_ms": tm, "precision": table,
        "tensor_peak": {"bf16_tflops": peaks["bf16_tflops"], "source": "MEASURED_PEAKS.json (cuBLAS bf16 burst)"},
        "clocks": clk.summary(),
    }))
    return 0


def run_subjects(args):
    """Uneven-size batching: 8 subjects with N = 68, 68, 100, 100, 200, 200,
    400, 400 (own seeded SC each, 30 % density, seeds 0..7), 64 CMA-ES
    particles per subject (512 simulations per generation), 300 s at TR 1 s,
    window 44 step 1, 30 s removed, FIC on.  Every generation is one CUDA graph
    launch over all subjects (bnm_group_run), each subject's integrator picked
    by the autotuner for its N (register kernel and particles per CTA for
    N <= 128, cluster size / nodes per warp / SC chunks in registers above).
    The first generation runs eagerly (tuning, graph capture) and is reported
    apart; sims/s is over the --subject-generations - 1 graph launches after it."""
    import bnm_cuda_b200 as B
    from bnm_cuda_b200 import synth
    from bnm_cuda_b200.surrogate import Bounds

    nodes, lam, T = [68, 68, 100, 100, 200, 200, 400, 400], 64, 300_000
    gens = max(2, args.subject_generations)
    bounds = Bounds()
    plans, cms = [], []
    for k, N in enumerate(nodes):
        sc = synth.make_sc(N, 0.3, k)
        cfg = B.Config(nodes=N, max_sims=lam, time_steps=T, bold_tr=1000, window_size=WS, window_step=1,
                       bold_remove_s=REMOVE_S, noise_seed=410)
        s = cfg.sizes()
        tcfg = B.Config(**{**cfg.__dict__, "max_sims": 1, "noise_seed": 1})
        with B.Plan(tcfg, sc, np.zeros(s["n_pairs"]), np.zeros(s["n_fcd"])) as tp:
            tr = tp.run(2.0, 0.3, 0.2, outputs=("fc", "fcd"))
        plans.append(B.Plan(cfg, sc, tr["fc"][0], tr["fcd"][0]))
        cms.append(B.CMAES(lam, 3, 1 + k, gens + 1, from_env=False))
    gen_ms, walls, graph, best, trials = [], [], [], [np.inf] * len(nodes), []
    with ClockSampler(0) as clk, B.Group(plans) as g:
        for gen in range(gens):
            params = []
            for es, N in zip(cms, nodes):
                feas, _, _ = es.samples()
                Gv, we, wi = bounds.to_params(feas)
                params.append((Gv, np.repeat(we[:, None], N, 1), np.repeat(wi[:, None], N, 1)))
            t0 = time.perf_counter()
            res = g.run(params)
            walls.append(time.perf_counter() - t0)
            last = g.last()
            gen_ms.append(last["ms"])
            graph.append(last["graph"])
            trials.append([float(r["fic_ntrials"].mean()) for r in res])
            for k, (es, r) in enumerate(zip(cms, res)):
                cost = r["cost"] + r["fic_penalty"]
                best[k] = min(best[k], float(cost.min()))
                es.tell(cost)
        shapes = [p.integrator() for p in plans]
        launches = sum(p.gram_timing()["launches"] for p in plans)
        # the last generation's stage times per subject (events on each subject's stream, inside the graph:
        # a stage's time includes waiting for SMs that other subjects hold)
        subject_ms = [{k: round(float(v), 1) for k, v in p.timings().items()} for p in plans]
        max_trials = [int(r["fic_ntrials"].max()) for r in res]
    timed_ms, timed_wall = float(np.sum(gen_ms[1:])), float(np.sum(walls[1:]))
    n_timed = len(gen_ms) - 1
    print(json.dumps({
        "metric": "sims/s", "value": 512 * n_timed / (timed_ms / 1e3), "unit": "sims/s", "n_gpus": 1,
        "steps": n_timed, "warmup": 1, "ms_per_step": timed_ms / n_timed, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "uneven-subjects-N68-100-200-400x2-300s-lambda64", "nodes": nodes, "particles": lam,
                   "model_time_ms": T, "tr_ms": 1000, "window": WS, "step": 1, "generations": gens,
                   "integrators": [{"nodes": N, **sh} for N, sh in zip(nodes, shapes)],
                   "graph": "one CUDA graph launch per generation over 8 subject streams"},
        "e2e": {"value": 512 * n_timed / timed_wall, "unit": "sims/s",
                "h2d_bytes_per_step": sum(8 * (lam + 2 * lam * N) for N in nodes),
                "d2h_bytes_per_step": sum(8 * lam * (5 + N) + 12 * lam for N in nodes)},
        "gpu_launches": launches * n_timed,
        "generation_ms": gen_ms, "graph_launched": graph, "first_generation_eager_ms": gen_ms[0],
        "mean_fic_trials": trials[-1], "max_fic_trials": max_trials, "subject_stage_ms": subject_ms,
        "best_cost": best, "clocks": clk.summary(),
    }))
    for p in plans:
        p.close()
    return 0


def main():
    global N_SIMS, T_MS, WORKLOAD
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="generation", choices=["generation", "surrogate", "precision", "subjects"],
                    help="generation: one CMA-ES generation (headline); surrogate: screened vs plain CMA-ES; "
                         "precision: FC/FCD Gram arithmetic against FP64 at N=400; subjects: 8 subjects of "
                         "N = 68..400 in one graph per generation")
    ap.add_argument("--subject-generations", type=int, default=4, help="subjects: generations (first is eager)")
    ap.add_argument("--check-sims", type=int, default=4, help="precision: particles checked against FP64")
    ap.add_argument("--nodes", type=int, default=400, help="precision: profiling knob, node count (default 400)")
    ap.add_argument("--gram", default="bf16x3", choices=["f32", "bf16", "bf16x3"],
                    help="generation: FC/FCD Gram arithmetic")
    ap.add_argument("--train-sims", type=int, default=20_000)
    ap.add_argument("--epochs", type=int, default=60)
    ap.add_argument("--generations", type=int, default=60)
    ap.add_argument("--surrogate-seeds", type=int, default=5, help="surrogate: CMA-ES seeds compared")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline sample")
    ap.add_argument("--particles", type=int, default=N_SIMS,
                    help="profiling knob: particles per GPU (precision workload: particles, default 64)")
    ap.add_argument("--model-ms", type=int, default=T_MS,
                    help="profiling knob: model time per simulation (precision workload: default 600000)")
    ap.add_argument("--profile", action="store_true",
                    help="profiling knob: no integrator autotuning (BNM_B200_TUNE=0: the default shape, no timing "
                         "launches), so that a run's launch order is fixed: the target simulation's kernels, then "
                         "each step's")
    args = ap.parse_args()
    if args.profile:
        os.environ["BNM_B200_TUNE"] = "0"
    if args.particles != N_SIMS or args.model_ms != T_MS:
        N_SIMS, T_MS = args.particles, args.model_ms
        WORKLOAD = f"profiling-case-N100-{T_MS // 1000}s-x{N_SIMS}"
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "surrogate":
        return run_surrogate(args)
    if args.workload == "precision":
        return run_precision(args)
    if args.workload == "subjects":
        return run_subjects(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
