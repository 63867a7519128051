"""GPU parity of the batched form: uneven query windows on both strands in one
call, seeded on the device; every unit must equal the per-call output of the
oracle on the host seeder's words for that window."""
import numpy as np
import pytest

import oracle
from segalign_b200 import SeedFilter, build_sub_mat, host_revcomp, host_seeds, synth
from tests.helpers import compare_segments, small_workload

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup(built):
    w = small_workload()
    p = oracle.params()
    idx, pos = oracle.build_table(w.target, p)
    sf = SeedFilter()
    sf.initialize_interface(1)
    sf.generate_shape_pos("12of19")
    sf.initialize_processor(False, 250_000, 19, build_sub_mat(910), 910, 3000, False)
    sf.send_ref_write_request(w.target)
    sf.generate_seed_pos_table(None, 1, 19, 12)
    sf.send_query_write_request(w.query, 0)
    return dict(w=w, p=p, idx=idx, pos=pos, sf=sf, R=oracle.encode(w.target), Q=oracle.encode(w.query),
                QR=oracle.encode_rc(w.query), rctext=host_revcomp(w.query))


def _units(L, seed):
    ch = synth.loguniform_chunks(seed, L, 2_000, 250_000)
    units = []
    for (a, b) in ch.tolist():
        units.append((0, 0, a, b))
        units.append((0, 1, L - b, L - a))
    return units


def test_batch_units_match_per_call_oracle(setup):
    w, p, sf = setup["w"], setup["p"], setup["sf"]
    L = len(w.query) - 19
    units = _units(L, 103) + [(0, 0, 5, 5)]  # plus one empty window
    outs = sf.seed_and_filter_batch(units)
    assert len(outs) == len(units)
    total_hits = total_surv = 0
    for (buf, rev, a, b), got in zip(units, outs):
        text = setup["rctext"] if rev else w.query
        seeds = host_seeds(text, a, b)
        if len(seeds) == 0:
            assert len(got) == 1 and int(got[0]["len"]) == 0 and int(got[0]["score"]) == 0
            continue
        want, st = oracle.seed_and_filter(p, setup["R"], setup["QR"] if rev else setup["Q"], setup["idx"],
                                          setup["pos"], seeds, rev)
        compare_segments(got, want, f"unit {(rev, a, b)}")
        total_hits += st["num_hits"]
        total_surv += st["survivors"]
    assert sf.last_call_stats()["num_hits"] == total_hits
    assert sf.last_call_stats()["survivors"] == total_surv


def test_batch_keep_on_device_counts(setup):
    sf = setup["sf"]
    L = len(setup["w"].query) - 19
    units = _units(L, 7)
    outs = sf.seed_and_filter_batch(units)
    st_out = sf.last_call_stats()
    sf.seed_and_filter_batch(units, keep_on_device=True)
    st_dev = sf.last_call_stats()
    assert st_dev["num_hits"] == st_out["num_hits"]
    assert st_dev["num_hsps"] == st_out["num_hsps"] == sum(len(o) - 1 for o in outs)


def test_batch_max_hits_iterations(setup):
    w, p, sf = setup["w"], setup["p"], setup["sf"]
    sf.set_max_hits(4000)
    try:
        units = [(0, 0, 0, 250_000), (0, 1, 100_000, 300_000), (0, 0, 600_000, 640_000)]
        outs = sf.seed_and_filter_batch(units)
        p2 = oracle.params(max_hits=4000)
        for (buf, rev, a, b), got in zip(units, outs):
            text = setup["rctext"] if rev else w.query
            seeds = host_seeds(text, a, b)
            want, st = oracle.seed_and_filter(p2, setup["R"], setup["QR"] if rev else setup["Q"], setup["idx"],
                                              setup["pos"], seeds, rev)
            assert st["num_iter"] > 1 or st["num_hits"] < 4000
            compare_segments(got, want, f"unit {(rev, a, b)} MAX_HITS=4000")
    finally:
        sf.set_max_hits(0)
