"""The oracle and the product against the reference's own SeedAndFilter.

tests/golden/ref_calls.npz holds outputs of the reference's seed-filter code
(src/seed_filter.cu:654-778 and repeat_masker_src/seed_filter.cu:723-855,
compiled unmodified for sm_100a and run on a B200 by
tests/golden/make_ref_golden.py) over the cases of tests/ref_cases.py:
every call's full HSP list, header included, under default parameters,
MAX_HITS iterations, transitions, the exact X-drop form (xdrop 500), entropy
off, and repeat-masker windows on both strands.  The CPU tests pin the oracle
to them bit for bit; the GPU test pins the product to them through the C ABI.
"""
import json
import os

import numpy as np
import pytest

from tests import ref_cases
from tests.helpers import compare_segments

FIX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_calls.npz")


@pytest.fixture(scope="module")
def recorded(built):
    arr = np.load(FIX)
    meta = {m["name"]: m for m in json.loads(arr["meta_json"].tobytes().decode())}
    cases = ref_cases.fixture_cases()
    for c in cases:
        m = meta[c["name"]]
        assert m["digest"] == c["digest"], f"{c['name']}: inputs differ from the ones the fixture was recorded on"
        assert m["ncalls"] == len(c["calls"])
    return arr, meta, cases


def _want(arr, name, k):
    return arr[f"{name}_{k}"].reshape(-1).view(ref_cases.oracle.SEGMENT_DTYPE)


def test_oracle_matches_reference_fixtures(recorded):
    arr, meta, cases = recorded
    total_hsps = 0
    for case in cases:
        for k, (segs, st) in enumerate(ref_cases.oracle_run(case)):
            want = _want(arr, case["name"], k)
            compare_segments(segs, want, f"{case['name']} call {k}")
            assert st["num_hits"] == meta[case["name"]]["num_hits"][k]
            assert st["num_seeds"] == meta[case["name"]]["num_seeds"][k]
            total_hsps += len(want) - 1
    assert total_hsps > 10_000


def test_fixture_covers_iterations_and_both_strands(recorded):
    arr, meta, cases = recorded
    mh = next(c for c in cases if c["name"] == "plain_max_hits_800")
    assert max(st["num_iter"] for _, st in ref_cases.oracle_run(mh)) > 1
    for name in ("plain_250k", "rm_acgt"):
        revs = {c["rev"] for c in next(c for c in cases if c["name"] == name)["calls"]}
        assert revs == {0, 1}


@pytest.mark.gpu
def test_gpu_matches_reference_fixtures(recorded):
    arr, meta, cases = recorded
    for case in cases:
        for k, got in enumerate(ref_cases.product_run(case)):
            compare_segments(got, _want(arr, case["name"], k), f"{case['name']} call {k}")
