"""Shared helpers of the parity tests: workloads, oracle runs, comparisons."""
from __future__ import annotations

import numpy as np

import oracle
from segalign_b200 import synth

SEG = oracle.SEGMENT_DTYPE


def compare_segments(got: np.ndarray, want: np.ndarray, what: str = "") -> None:
    """Bit-exact comparison of two HSP lists (header included)."""
    got = np.asarray(got, dtype=SEG)
    want = np.asarray(want, dtype=SEG)
    if len(got) == len(want) and np.array_equal(got.view(np.uint32).reshape(-1, 4), want.view(np.uint32).reshape(-1, 4)):
        return
    n = min(len(got), len(want))
    gv = got.view(np.uint32).reshape(-1, 4)[:n]
    wv = want.view(np.uint32).reshape(-1, 4)[:n]
    bad = np.nonzero((gv != wv).any(axis=1))[0]
    first = bad[:5].tolist()
    raise AssertionError(
        f"{what}: HSP lists differ (len got {len(got)} want {len(want)}); first differing rows {first}: "
        f"got {[tuple(got[i]) for i in first]} want {[tuple(want[i]) for i in first]}")


def small_workload(scale: float = 1.0, seed: int = 101):
    """The 1 Mbp x 1 Mbp plain-method workload (GC 36%, 200 inserted segments)."""
    return synth.make(1, seed=seed, scale=scale)


def random_text(rng: np.random.Generator, n: int, gc: float = 0.36, lower: float = 0.0, nfrac: float = 0.0) -> bytes:
    p = [(1 - gc) / 2, gc / 2, gc / 2, (1 - gc) / 2]
    a = rng.choice(np.frombuffer(b"ACGT", dtype=np.uint8), size=n, p=p)
    if lower:
        m = rng.random(n) < lower
        a[m] = a[m] + 32
    if nfrac:
        a[rng.random(n) < nfrac] = ord("N")
    return a.tobytes()
