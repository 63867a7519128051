"""Seeded synthetic genomes with the shapes of the benchmark workloads.

Thin binding over libsa_synth.so (segalign_b200/csrc/synth.cpp).  Stand-ins
for the genome assemblies the reference is run on; no dataset is needed.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
SYNTH_PATH = os.path.join(_HERE, "libsa_synth.so")
_lib = None

# config -> default seed (the workloads are named by their sizes in callers)
DEFAULT_SEEDS = {1: 101, 2: 102, 4: 104}


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(SYNTH_PATH):
            raise RuntimeError(f"{SYNTH_PATH} missing: run `python -m segalign_b200._build`")
        lib = C.CDLL(SYNTH_PATH)
        lib.synth_make.restype = C.c_void_p
        lib.synth_make.argtypes = [C.c_int, C.c_uint64, C.c_double]
        lib.synth_make_block.restype = C.c_void_p
        lib.synth_make_block.argtypes = [C.c_int, C.c_uint64, C.c_double, C.c_uint32]
        lib.synth_len.restype = C.c_uint64
        lib.synth_len.argtypes = [C.c_void_p, C.c_int]
        lib.synth_copy.restype = None
        lib.synth_copy.argtypes = [C.c_void_p, C.c_int, C.c_char_p]
        lib.synth_nchr.restype = C.c_uint32
        lib.synth_nchr.argtypes = [C.c_void_p, C.c_int]
        lib.synth_chr.restype = None
        lib.synth_chr.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
        lib.synth_free.restype = None
        lib.synth_free.argtypes = [C.c_void_p]
        lib.synth_chunks.restype = C.c_uint32
        lib.synth_chunks.argtypes = [C.c_uint64, C.c_uint64, C.c_double, C.c_double, C.POINTER(C.c_uint64), C.c_uint32]
        _lib = lib
    return _lib


class Workload:
    """target / query block texts (bytes) and their chromosome (start, length) tables."""

    def __init__(self, target: bytes, query: bytes, tchr, qchr):
        self.target, self.query, self.target_chr, self.query_chr = target, query, tchr, qchr


def make(config: int, seed: int | None = None, scale: float = 1.0, block: int = 0) -> Workload:
    """config 1: 1 Mbp x 1 Mbp; 2: 100 Mbp (6 chr) x 108 Mbp; 4: 600 Mbp (12 chr) x 600 Mbp.

    block > 0 (configs 2 and 4): the same target with another query block of the
    same size, drawn from that target the same way (one job's query in blocks)."""
    lib = _load()
    h = lib.synth_make_block(config, DEFAULT_SEEDS.get(config, 1) if seed is None else seed, scale, block)
    if not h:
        raise ValueError(f"unknown workload config {config} (block {block})")
    try:
        out = []
        chrs = []
        for which in (0, 1):
            n = lib.synth_len(h, which)
            buf = C.create_string_buffer(n)
            lib.synth_copy(h, which, buf)
            out.append(buf.raw[:n])
            k = lib.synth_nchr(h, which)
            st = (C.c_uint64 * k)()
            ln = (C.c_uint64 * k)()
            lib.synth_chr(h, which, st, ln)
            chrs.append(list(zip(list(st), list(ln))))
        return Workload(out[0], out[1], chrs[0], chrs[1])
    finally:
        lib.synth_free(h)


def loguniform_chunks(seed: int, length: int, lo: float, hi: float) -> np.ndarray:
    """[start, end) windows covering [0, length) with log-uniform lengths in [lo, hi]."""
    lib = _load()
    n = lib.synth_chunks(seed, length, lo, hi, None, 0)
    b = (C.c_uint64 * (2 * n))()
    lib.synth_chunks(seed, length, lo, hi, b, n)
    return np.array(list(b), dtype=np.uint64).reshape(n, 2)
