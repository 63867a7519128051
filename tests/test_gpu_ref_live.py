"""Live three-way parity: the reference's own SeedAndFilter (compiled unmodified
for sm_100a, oracle/ref_harness.cu) == the CPU oracle == the product, bit for
bit, header included, on the 1 Mbp x 1 Mbp workload (every 250 kbp call on
both strands), with transitions, with MAX_HITS iterations, and in
repeat-masker mode on a 1.8 Mbp repeat-rich sequence.

Inputs pass through oracle.ref_safe_texts / ref_filter_seeds so that the
reference's kernel stays clear of its undefined behaviour (see
oracle/ref_harness.cu); the cases are otherwise the workload's own.
"""
import numpy as np
import pytest

import oracle
from segalign_b200 import synth
from tests import ref_cases
from tests.helpers import compare_segments

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (oracle.ref_harness_available("plain") and oracle.ref_harness_available("rm")),
                                 reason="reference harness not built (make -C oracle ref_kernels needs the reference tree)")]


def _three_way(case):
    ref = ref_cases.reference_run(case)
    orc = ref_cases.oracle_run(case)
    prod = ref_cases.product_run(case)
    hits = hsps = 0
    for k, (r, (o, st), g) in enumerate(zip(ref, orc, prod)):
        compare_segments(o, r["segments"], f"{case['name']} call {k}: oracle vs reference")
        compare_segments(g, r["segments"], f"{case['name']} call {k}: product vs reference")
        assert r["num_seeds"] == len(case["calls"][k]["seeds"])
        hits += st["num_hits"]
        hsps += len(o) - 1
    secs = sum(r["seconds"] for r in ref)
    print(f"{case['name']}: {len(ref)} calls, {hits} hits, {hsps} HSPs, reference {secs:.3f} s")
    return hits, hsps


@pytest.fixture(scope="module")
def one_mbp(built):
    w = synth.make(1, seed=101)
    return oracle.ref_safe_texts(w.target, w.query)


def test_reference_one_mbp_every_call(one_mbp):
    T, Q = one_mbp
    p = oracle.params()
    case = {"name": "1Mbp", "mode": "plain", "kw": {}, "target": T, "query": Q,
            "calls": ref_cases._plain_calls(T, Q, p, 250_000)}
    assert len(case["calls"]) == 8
    hits, hsps = _three_way(case)
    assert hits > 250_000 and hsps > 100


def test_reference_one_mbp_max_hits(one_mbp):
    T, Q = one_mbp
    p = oracle.params()
    case = {"name": "1Mbp_max_hits", "mode": "plain", "kw": {"max_hits": 3000}, "target": T, "query": Q,
            "calls": ref_cases._plain_calls(T, Q, p, 250_000, j_hi=250_000)}
    _three_way(case)
    assert max(st["num_iter"] for _, st in ref_cases.oracle_run(case)) > 5


def test_reference_one_mbp_transitions(one_mbp):
    T, Q = one_mbp
    p = oracle.params(transition=True)
    case = {"name": "1Mbp_transition", "mode": "plain", "kw": {"transition": True}, "target": T, "query": Q,
            "calls": ref_cases._plain_calls(T, Q, p, 100_000, j_lo=400_000, j_hi=600_000)}
    hits, _ = _three_way(case)
    assert hits > 200_000


def test_reference_repeat_masker_windows(built):
    S = ref_cases.acgt_only(synth.make(4, seed=11, scale=0.003).target)
    p = oracle.params()
    n = len(S)
    ranges = [(600_000, 700_000), (100_000, 200_000), (1_300_000, 1_400_000)]
    windows = [(200_000, 560_000), (250_000, 900_000), (200_000, 1_250_000)]
    case = {"name": "rm_1.8Mbp", "mode": "rm", "kw": {}, "target": S, "query": None,
            "calls": ref_cases._rm_calls(S, p, ranges, windows)}
    hits, hsps = _three_way(case)
    assert hsps > 1000
