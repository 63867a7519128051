"""Builds the native libraries of segalign_b200 in-tree.

  segalign_b200/libsegalign_b200.so  CUDA kernels + C ABI (nvcc, sm_100a)
  segalign_b200/libsa_synth.so       synthetic genome generator (g++)

Usage: python -m segalign_b200._build [--force]
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_obj")
LIB = os.path.join(HERE, "libsegalign_b200.so")
SYNTH = os.path.join(HERE, "libsa_synth.so")

CU_SOURCES = ["sa_pack.cu", "sa_lookup.cu", "sa_extend.cu", "sa_sort.cu", "sa_api.cu", "sa_host.cpp", "sa_noalloc.cu", "sa_serve.cu", "sa_tune.cu",
              "sa_ingest.cpp", "sa_coverage.cu", "sa_segwrite.cu"]
HEADERS = ["sa_internal.cuh", "sa_launch.h", "sa_radix.cuh", "sa_host_internal.h", "sa_slot_pool.h"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    "--expt-relaxed-constexpr",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"command failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def build(force: bool = False, verbose: bool = False, extra_flags: list[str] | None = None) -> str:
    os.makedirs(OBJ, exist_ok=True)
    nvcc = _nvcc()
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [
        os.path.join(HERE, "..", "include", h) for h in ("segalign_b200.h", "segalign_b200_host.h")]
    jobs = []
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            cmd = [nvcc] + NVCC_FLAGS + (extra_flags or []) + ["-c", s, "-o", o]
            jobs.append(cmd)
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as ex:
            list(ex.map(_run, jobs))
    if force or jobs or _stale(LIB, objs):
        _run([nvcc, "-shared", "-o", LIB] + objs + ["-lcudart", "-lz"])
    synth_src = os.path.join(CSRC, "synth.cpp")
    if force or _stale(SYNTH, [synth_src]):
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-o", SYNTH, synth_src])
    if verbose:
        print("built", LIB, SYNTH)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
