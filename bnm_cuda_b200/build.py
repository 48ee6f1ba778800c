"""Builds the library in-tree: ``bnm_cuda_b200/libbnm_b200.so`` (CUDA kernels for
sm_100a + host C/C++ ABI) and the drop-in CLI ``bnm_cuda_b200/run_CMAES_gpu``.

    python -m bnm_cuda_b200.build [--force]

Every .cu is compiled by nvcc for ``-gencode arch=compute_100a,code=sm_100a``;
integrate_exact.cu additionally with ``-fmad=false`` (reference-order
arithmetic, no FMA contraction).  Host C++ is compiled by the system g++ so
that its <random> engines are the same libstdc++ ones the reference uses.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libbnm_b200.so")
CLI = os.path.join(HERE, "run_CMAES_gpu")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
HOSTCXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")

CU = {
    "integrate_fast.cu": [],
    "integrate_exact.cu": ["-fmad=false"],
    "analysis.cu": [],
    "fic_noise.cu": [],
    "capi.cu": [],
    "probe.cu": [],
    "noalloc.cu": [],
    "mlp.cu": [],
    "gram_tc.cu": [],
    "integrate_cluster.cu": [],
    "integrate_colsplit.cu": [],
}
CPP = ["cmaes.cpp", "params.cpp"]
HEADERS = ["bnm_common.cuh", "integrate_generic.cuh", "kernels.h", "fp32_model.cuh", "cluster_util.cuh",
           "noise.cuh"]


def _newer(src_paths, out):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(p) > t for p in src_paths)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build step failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(HERE, "..", "include", "bnm_b200.h")]
    jobs, objs = [], []
    ccbin = ["-ccbin", HOSTCXX]
    for f, extra in CU.items():
        src, obj = os.path.join(CSRC, f), os.path.join(OBJ, f + ".o")
        objs.append(obj)
        if force or _newer([src] + hdrs, obj):
            jobs.append([NVCC, *ccbin, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", *extra, "-c",
                         src, "-o", obj])
    for f in CPP:
        src, obj = os.path.join(CSRC, f), os.path.join(OBJ, f + ".o")
        objs.append(obj)
        if force or _newer([src] + hdrs, obj):
            jobs.append([HOSTCXX, "-O2", "-std=c++17", "-fPIC", "-c", src, "-o", obj])
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for r in ex.map(_run, jobs):
            if verbose and (r.stdout or r.stderr):
                print(r.stdout, r.stderr)
    if force or jobs or not os.path.exists(LIB):
        _run([NVCC, *ccbin, *ARCH, "-shared", "-o", LIB, *objs, "-Xlinker", "-rpath,$ORIGIN"])
    cli_src = os.path.join(CSRC, "run_cmaes_main.cpp")
    if os.path.exists(cli_src) and (force or _newer([cli_src, LIB] + hdrs, CLI)):
        _run([HOSTCXX, "-O2", "-std=c++17", cli_src, "-o", CLI, f"-L{HERE}", "-lbnm_b200", "-Wl,-rpath,$ORIGIN"])
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
