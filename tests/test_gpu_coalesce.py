"""GPU tests of call coalescing: sa_seed_and_filter calls made concurrently
share device passes (batch_calls > 1 in their stats) and each still gets,
bit for bit, the HSP list the oracle gives for that call alone, MAX_HITS
iterations included; a call with a bad seed key in a shared pass fails
alone with the plain path's status while the others complete."""
import os
import threading

import numpy as np
import pytest

import oracle
from segalign_b200 import SeedFilter, SegAlignError, build_sub_mat, host_revcomp, host_seeds
from tests.helpers import compare_segments, small_workload

pytestmark = pytest.mark.gpu

CHUNK = 50_000


@pytest.fixture(scope="module")
def setup(built):
    w = small_workload()
    p = oracle.params()
    idx, pos = oracle.build_table(w.target, p)
    sf = SeedFilter()
    sf.initialize_interface(1)
    sf.generate_shape_pos("12of19")
    # one slot: concurrent calls queue behind it and are taken as one pass
    old = {k: os.environ.get(k) for k in ("SA_SLOTS_PER_GPU", "SA_COALESCE")}
    os.environ["SA_SLOTS_PER_GPU"] = "1"
    os.environ["SA_COALESCE"] = "16"
    try:
        sf.initialize_processor(False, CHUNK, 19, build_sub_mat(910), 910, 3000, False)
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    sf.send_ref_write_request(w.target)
    sf.generate_seed_pos_table(None, 1, 19, 12)
    sf.send_query_write_request(w.query, 0)
    rct = host_revcomp(w.query)
    L = len(w.query) - 19
    calls = [(rev, j0, min(j0 + CHUNK, L)) for rev in (0, 1) for j0 in range(0, L, 3 * CHUNK)]
    seeds = [host_seeds(rct if rev else w.query, a, b) for (rev, a, b) in calls]
    R, Q, QR = oracle.encode(w.target), oracle.encode(w.query), oracle.encode_rc(w.query)
    want = [oracle.seed_and_filter(p, R, QR if rev else Q, idx, pos, s, bool(rev)) for (rev, _, _), s in
            zip(calls, seeds)]
    yield dict(sf=sf, calls=calls, seeds=seeds, want=want, p=p, R=R, Q=Q, QR=QR, idx=idx, pos=pos)
    sf.initialize_processor(False, CHUNK, 19, build_sub_mat(910), 910, 3000, False)


def _concurrent(sf, jobs):
    """Runs (seeds, rev) jobs from one thread each, all released together."""
    out, stats, errs = [None] * len(jobs), [None] * len(jobs), [None] * len(jobs)
    gate = threading.Barrier(len(jobs))

    def run(i):
        s, rev = jobs[i]
        gate.wait()
        try:
            out[i] = sf.seed_and_filter(s, rev, 0)
            stats[i] = sf.last_call_stats()
        except SegAlignError as e:
            errs[i] = e

    th = [threading.Thread(target=run, args=(i,)) for i in range(len(jobs))]
    for t in th:
        t.start()
    for t in th:
        t.join()
    return out, stats, errs


def test_calls_alone_match_oracle(setup):
    sf = setup["sf"]
    for (rev, a, _), s, (want, st) in zip(setup["calls"], setup["seeds"], setup["want"]):
        compare_segments(sf.seed_and_filter(s, bool(rev), 0), want, f"alone rev={rev} j0={a}")
        cs = sf.last_call_stats()
        assert cs["batch_calls"] == 1
        assert cs["num_hits"] == st["num_hits"] and cs["tiles"] == st["tiles_right"] + st["tiles_left"]


def test_concurrent_calls_share_passes_and_match_oracle(setup):
    sf = setup["sf"]
    jobs = [(s, bool(rev)) for (rev, _, _), s in zip(setup["calls"], setup["seeds"])]
    shared = 0
    for rep in range(3):
        out, stats, errs = _concurrent(sf, jobs)
        assert not any(errs), errs
        for i, ((rev, a, _), (want, st)) in enumerate(zip(setup["calls"], setup["want"])):
            compare_segments(out[i], want, f"concurrent rep {rep} rev={rev} j0={a}")
            assert stats[i]["num_hits"] == st["num_hits"] and stats[i]["num_seeds"] == len(jobs[i][0])
            assert stats[i]["num_hsps"] == len(want) - 1
        shared = max(shared, max(s["batch_calls"] for s in stats))
    assert shared > 1, "no two calls shared a device pass"


def test_iterations_in_a_shared_pass(setup):
    """Small MAX_HITS: every call of a shared pass keeps its own iterations."""
    sf, p = setup["sf"], setup["p"]
    p2 = oracle.params(max_hits=4000)
    sf.set_max_hits(4000)
    try:
        jobs = [(s, bool(rev)) for (rev, _, _), s in zip(setup["calls"], setup["seeds"])]
        out, stats, errs = _concurrent(sf, jobs)
        assert not any(errs), errs
        for i, ((rev, a, _), s) in enumerate(zip(setup["calls"], setup["seeds"])):
            want, st = oracle.seed_and_filter(p2, setup["R"], setup["QR"] if rev else setup["Q"], setup["idx"],
                                              setup["pos"], s, bool(rev))
            compare_segments(out[i], want, f"MAX_HITS 4000 rev={rev} j0={a}")
            assert stats[i]["num_iter"] == st["num_iter"]
        assert max(st["num_iter"] for st in stats) > 1
    finally:
        sf.set_max_hits(0)


def test_bad_call_fails_alone_in_a_shared_pass(setup):
    sf = setup["sf"]
    jobs = [(s, bool(rev)) for (rev, _, _), s in zip(setup["calls"], setup["seeds"])]
    bad = jobs[2][0].copy()
    bad[len(bad) // 2] = (np.uint64(1 << 24) << np.uint64(32)) | np.uint64(7)  # key outside the 4^12 table
    jobs[2] = (bad, jobs[2][1])
    out, stats, errs = _concurrent(sf, jobs)
    assert errs[2] is not None and errs[2].code == -6  # SA_ERR_BAD_SEED
    for i, ((rev, a, _), (want, _)) in enumerate(zip(setup["calls"], setup["want"])):
        if i != 2:
            assert errs[i] is None, errs[i]
            compare_segments(out[i], want, f"beside a bad call rev={rev} j0={a}")
