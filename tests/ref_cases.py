"""Inputs on which the reference's own SeedAndFilter is run (oracle/ref_harness.cu).

Shared by tests/golden/make_ref_golden.py (which records the reference's
outputs as fixtures on a GPU) and by the tests that replay them.  Every input
satisfies the harness's safety preconditions:
  * plain mode: the target carries no N and the query no lowercase
    (oracle.ref_safe_texts), so no code >= 4 occurs on both sides;
  * repeat-masker mode: the sequence is ACGT only, and the ref windows avoid
    the seeds' own diagonal (a self hit on an ACGT-only sequence would extend to
    the sequence end);
  * seeds whose hits could start a tile past a sequence end are dropped
    (oracle.ref_filter_seeds).
"""
from __future__ import annotations

import hashlib

import numpy as np

import oracle
from segalign_b200 import synth

SEED_SIZE = 19


def acgt_only(text: bytes, fill: int = ord("G")) -> bytes:
    """Uppercase, separators removed, N replaced by `fill`."""
    a = np.frombuffer(text.upper().replace(b"&", b""), dtype=np.uint8).copy()
    a[a == ord("N")] = fill
    return a.tobytes()


def _plain_calls(T: bytes, Q: bytes, p, chunk: int, j_lo: int = 0, j_hi: int | None = None, strands=(0, 1)):
    tk = oracle.ref_tail_keys(T, p)
    rct = oracle.revcomp_text(Q)
    L = len(Q) - SEED_SIZE if j_hi is None else j_hi
    calls = []
    for rev in strands:
        text = rct if rev else Q
        for j0 in range(j_lo, L, chunk):
            s = oracle.ref_filter_seeds(oracle.chunk_seeds(text, j0, min(j0 + chunk, L), p), tk, len(Q))
            if len(s):
                calls.append({"rev": rev, "seeds": s, "j0": j0})
    return calls


def _rm_calls(S: bytes, p, seed_ranges, windows):
    tk = oracle.ref_tail_keys(S, p)
    rct = oracle.revcomp_text(S)
    calls = []
    for (j0, j1), (rs, re_) in zip(seed_ranges, windows):
        for rev in (0, 1):
            text = rct if rev else S
            s = oracle.ref_filter_seeds(oracle.chunk_seeds(text, j0, j1, p), tk, len(S))
            if len(s):
                calls.append({"rev": rev, "seeds": s, "j0": j0, "ref_start": rs, "ref_end": re_})
    return calls


def case_inputs_digest(case) -> str:
    h = hashlib.sha256()
    h.update(case["target"])
    h.update(case.get("query") or b"")
    for c in case["calls"]:
        h.update(np.ascontiguousarray(c["seeds"], dtype="<u8").tobytes())
        h.update(bytes([c["rev"]]))
    return h.hexdigest()


def fixture_cases():
    """Small cases recorded as committed fixtures (tests/golden/ref_calls.npz)."""
    w = synth.make(1, seed=4242, scale=0.25)
    T, Q = oracle.ref_safe_texts(w.target, w.query)
    out = []
    p = oracle.params()
    out.append({"name": "plain_250k", "mode": "plain", "kw": {}, "target": T, "query": Q,
                "calls": _plain_calls(T, Q, p, 25_000)})
    out.append({"name": "plain_max_hits_800", "mode": "plain", "kw": {"max_hits": 800}, "target": T, "query": Q,
                "calls": _plain_calls(T, Q, p, 50_000, j_hi=100_000)})
    pt = oracle.params(transition=True)
    out.append({"name": "plain_transition", "mode": "plain", "kw": {"transition": True}, "target": T, "query": Q,
                "calls": _plain_calls(T, Q, pt, 20_000, j_hi=60_000)})
    out.append({"name": "plain_xdrop500_h1500", "mode": "plain", "kw": {"xdrop": 500, "hspthresh": 1500},
                "target": T, "query": Q, "calls": _plain_calls(T, Q, p, 40_000, j_hi=120_000)})
    out.append({"name": "plain_noentropy", "mode": "plain", "kw": {"noentropy": True}, "target": T, "query": Q,
                "calls": _plain_calls(T, Q, p, 40_000, j_hi=120_000)})
    S = acgt_only(synth.make(4, seed=11, scale=0.0005).target)
    out.append({"name": "rm_acgt", "mode": "rm", "kw": {}, "target": S, "query": None,
                "calls": _rm_calls(S, p, [(150_000, 200_000), (10_000, 40_000)],
                                   [(20_000, 120_000), (60_000, 250_000)])})
    for c in out:
        c["digest"] = case_inputs_digest(c)
    return out


def oracle_run(case):
    """The oracle's per-call outputs for a case (header row first)."""
    kw = dict(case["kw"])
    max_hits = kw.pop("max_hits", 0)
    p = oracle.params(max_hits=max_hits or (1 << 40), **kw)
    T = case["target"]
    rm = case["mode"] == "rm"
    Qt = T if rm else case["query"]
    idx, pos = oracle.build_table(T, p)
    R = oracle.encode(T)
    qf = R if rm else oracle.encode(Qt)
    qr = oracle.rc_codes(R) if rm else oracle.encode_rc(Qt)
    outs = []
    for c in case["calls"]:
        segs, st = oracle.seed_and_filter(p, R, qr if c["rev"] else qf, idx, pos, c["seeds"], bool(c["rev"]),
                                          1 if rm else 0, c.get("ref_start", 0), c.get("ref_end", 0))
        outs.append((segs, st))
    return outs


def product_run(case):
    """The product's per-call outputs for a case, through the C ABI."""
    from segalign_b200 import SeedFilter, build_sub_mat

    kw = case["kw"]
    xdrop, hsp = kw.get("xdrop", 910), kw.get("hspthresh", 3000)
    rm = case["mode"] == "rm"
    sf = SeedFilter()
    sf.initialize_interface(1)
    sf.generate_shape_pos("12of19")
    sf.initialize_processor(bool(kw.get("transition", False)), 250_000, SEED_SIZE, build_sub_mat(xdrop), xdrop, hsp,
                            bool(kw.get("noentropy", False)))
    sf.send_ref_write_request(case["target"])
    sf.generate_seed_pos_table(None, 1, SEED_SIZE, 12)
    if rm:
        sf.rm_send_query_write_request()
    else:
        sf.send_query_write_request(case["query"], 0)
    if kw.get("max_hits"):
        sf.set_max_hits(kw["max_hits"])
    try:
        outs = []
        for c in case["calls"]:
            if rm:
                outs.append(sf.rm_seed_and_filter(c["seeds"], bool(c["rev"]), c["ref_start"], c["ref_end"]))
            else:
                outs.append(sf.seed_and_filter(c["seeds"], bool(c["rev"]), 0))
        return outs
    finally:
        sf.set_max_hits(0)
        sf.shutdown_processor()


def reference_run(case, records: bool = True):
    """The reference's own SeedAndFilter over a case (needs a GPU)."""
    kw = case["kw"]
    return oracle.ref_seed_and_filter(case["calls"], case["target"], case.get("query"), mode=case["mode"],
                                      records=records, wga_chunk=250_000, **kw)
