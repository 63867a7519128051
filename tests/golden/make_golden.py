"""Regenerates the golden fixtures of tests/golden/ from the CPU oracle.

The reference ships no tests or golden vectors, so these fixtures are
produced by the oracle (oracle/sa_oracle.cpp, a restatement of the reference
semantics) on seeded inputs and committed; the hand-derived known-answer
tests live in tests/test_oracle_kat.py.  Run from the repository root:

    python tests/golden/make_golden.py            # every fixture
    python tests/golden/make_golden.py --rm-only  # the repeat-masker runs only (slow: oracle)
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from segalign_b200 import synth  # noqa: E402

CHUNK = 20_000


def kat_cases(rng):
    """Single hits on short planted alignments: edges, N/lowercase/separators, entropy branch."""
    cases = []
    alph = np.frombuffer(b"ACGT", dtype=np.uint8)
    for k in range(48):
        n = int(rng.integers(60, 400))
        R = rng.choice(alph, size=n)
        Q = R.copy()
        sub = rng.random(n) < rng.choice([0.05, 0.15, 0.3])
        Q[sub] = rng.choice(alph, size=int(sub.sum()))
        if k % 4 == 1:
            R[rng.integers(0, n)] = ord("N")
        if k % 4 == 2:
            i = int(rng.integers(0, n - 20))
            R[i:i + 10] += 32
        if k % 4 == 3:
            Q[int(rng.integers(0, n))] = ord("&")
        if k % 6 == 0:  # low-complexity run -> entropy branch
            i = int(rng.integers(0, n // 2))
            R[i:i + 40] = ord("A")
            Q[i:i + 40] = ord("A")
        rl = int(rng.integers(19, n))
        ql = int(rng.integers(19, n)) if k % 5 == 4 else rl
        p = {"xdrop": int(rng.choice([910, 500, 200])), "hspthresh": int(rng.choice([3000, 1500, 500])),
             "noentropy": bool(k % 7 == 6)}
        P = oracle.params(**p)
        Rb, Qb = R.tobytes(), Q.tobytes()
        r = oracle.extend_hit(P, oracle.encode(Rb), oracle.encode(Qb), rl, ql)
        cases.append({"R": Rb.decode(), "Q": Qb.decode(), "ref_loc": rl, "query_loc": ql, "params": p,
                      "expect": {k2: r[k2] for k2 in ("right_best", "right_pos", "left_best", "left_pos", "total",
                                                      "keep", "score", "entropy_branch")}})
    return cases


def small_calls():
    w = synth.make(1, seed=4242, scale=0.05)
    T, Qt = w.target, w.query
    p = oracle.params()
    idx, pos = oracle.build_table(T, p)
    R, Q, QR = oracle.encode(T), oracle.encode(Qt), oracle.encode_rc(Qt)
    rc_text = oracle.revcomp_text(Qt)
    L = len(Qt) - 19
    out = {"target": np.frombuffer(T, dtype=np.uint8), "query": np.frombuffer(Qt, dtype=np.uint8)}
    calls = []
    for rev in (0, 1):
        text = rc_text if rev else Qt
        for j0 in range(0, L, CHUNK):
            j1 = min(j0 + CHUNK, L)
            seeds = oracle.chunk_seeds(text, j0, j1, p)
            segs, st = oracle.seed_and_filter(p, R, QR if rev else Q, idx, pos, seeds, rev)
            key = f"plain_{rev}_{j0}"
            out[key + "_out"] = segs.view(np.uint32).reshape(-1, 4)
            calls.append({"key": key, "rev": rev, "j0": j0, "j1": j1, "num_seeds": len(seeds),
                          "num_hits": st["num_hits"]})
    # repeat-masker self alignment of the target, window [5000, 40000]
    RC = oracle.rc_codes(R)
    t_rc = oracle.revcomp_text(T)
    for rev in (0, 1):
        text = t_rc if rev else T
        seeds = oracle.chunk_seeds(text, 10_000, 30_000, p)
        segs, st = oracle.seed_and_filter(p, R, RC if rev else R, idx, pos, seeds, rev, 1, 5000, 40000)
        key = f"rm_{rev}"
        out[key + "_out"] = segs.view(np.uint32).reshape(-1, 4)
        calls.append({"key": key, "rev": rev, "j0": 10_000, "j1": 30_000, "rm_ref_start": 5000, "rm_ref_end": 40000,
                      "num_seeds": len(seeds), "num_hits": st["num_hits"]})
    return out, calls


# Repeat-masker self-alignment fixture: a repeat-rich 1.8 Mbp sequence (the
# large workload's generator at scale 0.003, seed 11) in two blocks.
RM = dict(scale=0.003, seed=11, interval_size=300_000, block_size=1_200_000, prop=0.2, chunk=100_000)
RM_CASES = [(1, True), (2, False)]  # (M, diagonal excluded)


def rm_runs(seq: bytes, M: int, exclude: bool) -> np.ndarray:
    """The oracle's repeat-masker pipeline: block/interval plan
    (repeat_masker_src/main.cpp:319-428), rm SeedAndFilter per chunk and strand
    (repeat_masker_src/seeder.cpp:40-149), uint8 coverage runs (:151-186).
    Rows: block, interval, block-relative start, length."""
    isz, bsz, prop, ch = RM["interval_size"], RM["block_size"], RM["prop"], RM["chunk"]
    p = oracle.params(rm_exclude_diag=exclude)
    plan = oracle.rm_plan(len(seq), isz, bsz, prop)
    rc_all = oracle.revcomp_text(seq) + b"N" * 64  # minus-strand seeds near a block end read past it
    runs, tables = [], {}
    for k, (blk, b0, bl, s, e, rs, re_) in enumerate(plan.tolist()):
        block = seq[b0:b0 + bl]
        if blk not in tables:
            R = oracle.encode(block)
            tables[blk] = (oracle.build_table(block, p), R, oracle.rc_codes(R))
        (idx, pos), R, RC = tables[blk]
        rct = rc_all[len(seq) - b0 - bl:]
        hsps = []
        for i in range(s, e, ch):
            ee = min(i + ch, e)
            sd = oracle.chunk_seeds(block, i, ee, p)
            if len(sd):
                hsps.append(oracle.seed_and_filter(p, R, R, idx, pos, sd, False, 1, rs, re_)[0][1:])
            ms = bl - 1 - ee
            me = min(ms + ch, bl - 1 - s)
            if me > ms:
                sd = oracle.chunk_seeds(rct, ms, me, p)
                if len(sd):
                    hsps.append(oracle.seed_and_filter(p, R, RC, idx, pos, sd, True, 1, rs, re_)[0][1:])
        h = np.concatenate(hsps) if hsps else np.zeros(0, dtype=oracle.SEGMENT_DTYPE)
        st, ln = oracle.rm_intervals(h, bl, M)
        runs += [(blk, k, int(a), int(b)) for a, b in zip(st, ln)]
    return np.array(runs, dtype=np.uint32).reshape(-1, 4)


def rm_fixture():
    seq = synth.make(4, seed=RM["seed"], scale=RM["scale"]).target
    arrays = {f"M{M}_exclude{int(ex)}": rm_runs(seq, M, ex) for M, ex in RM_CASES}
    np.savez_compressed(os.path.join(HERE, "rm_runs.npz"), **arrays)
    with open(os.path.join(HERE, "rm_runs.json"), "w") as f:
        json.dump({**RM, "seq_len": len(seq), "cases": [list(c) for c in RM_CASES]}, f, indent=1)
    print("wrote rm runs", {k: len(v) for k, v in arrays.items()})


def main():
    if "--rm-only" not in sys.argv:
        small_fixtures()
    rm_fixture()


def small_fixtures():
    rng = np.random.default_rng(20261203)
    with open(os.path.join(HERE, "kat_cases.json"), "w") as f:
        json.dump(kat_cases(rng), f, indent=0)
    arrays, calls = small_calls()
    np.savez_compressed(os.path.join(HERE, "small_calls.npz"), **arrays)
    with open(os.path.join(HERE, "small_calls.json"), "w") as f:
        json.dump({"chunk": CHUNK, "calls": calls}, f, indent=1)
    print("wrote", len(calls), "calls")


if __name__ == "__main__":
    main()
