"""GPU parity: the sm_100a path through the C ABI against the CPU oracle.

Workload: the 1 Mbp x 1 Mbp plain-method configuration (seeded synthetic
stand-in), 12of19, HOXD70, xdrop 910, hspthresh 3000, entropy on, both
strands, 250 kbp WGA chunks.  Integer fields must match bit for bit.
"""
import numpy as np
import pytest

import oracle
from segalign_b200 import SeedFilter, build_sub_mat, host_revcomp, host_seeds, synth
from tests.helpers import compare_segments, small_workload, random_text

pytestmark = pytest.mark.gpu

CHUNK = 250_000


@pytest.fixture(scope="module")
def setup(built):
    w = small_workload()
    p = oracle.params()
    idx, pos = oracle.build_table(w.target, p)
    sf = SeedFilter()

    def restore():
        """(Re)loads this module's workload: other tests load their own
        targets into the same process-wide library state."""
        sf.initialize_interface(1)
        sf.generate_shape_pos("12of19")
        sf.initialize_processor(False, CHUNK, 19, build_sub_mat(910), 910, 3000, False)
        sf.send_ref_write_request(w.target)
        sf.generate_seed_pos_table(None, 1, 19, 12)
        sf.send_query_write_request(w.query, 0)

    restore()
    return dict(w=w, p=p, idx=idx, pos=pos, sf=sf, R=oracle.encode(w.target), Q=oracle.encode(w.query),
                QR=oracle.encode_rc(w.query), rctext=host_revcomp(w.query), restore=restore)


def test_device_table_matches_oracle(setup):
    it, pt = setup["sf"].get_seed_pos_table()
    assert np.array_equal(it, setup["idx"])
    assert np.array_equal(pt, setup["pos"])


@pytest.mark.parametrize("rev", [False, True])
def test_seed_and_filter_per_chunk(setup, rev):
    w, p, sf = setup["w"], setup["p"], setup["sf"]
    text = setup["rctext"] if rev else w.query
    qcodes = setup["QR"] if rev else setup["Q"]
    L = len(w.query) - 19
    total_hits = 0
    for j0 in range(0, L, CHUNK):
        j1 = min(j0 + CHUNK, L)
        seeds = host_seeds(text, j0, j1)
        assert np.array_equal(seeds, oracle.chunk_seeds(text, j0, j1, p))
        got = sf.seed_and_filter(seeds, rev, 0)
        want, st = oracle.seed_and_filter(p, setup["R"], qcodes, setup["idx"], setup["pos"], seeds, rev)
        compare_segments(got, want, f"chunk {j0} rev={rev}")
        cs = sf.last_call_stats()
        assert cs["num_hits"] == st["num_hits"]
        assert cs["tiles"] == st["tiles_right"] + st["tiles_left"]
        # kept HSPs before dedup: candidates already in the call's HSP set
        # count as kept without their keep test being rerun
        assert cs["survivors"] == st["survivors"]
        total_hits += st["num_hits"]
    assert total_hits > 100_000


def test_seeder_pipeline_matches_oracle(setup):
    w, p, sf = setup["w"], setup["p"], setup["sf"]
    fw, rc, st = sf.seeder_run(w.query, buffer=0, strand=3, num_threads=4)
    ofw, orc, ost = oracle.pipeline(p, w.target, w.query, setup["idx"], setup["pos"], nthreads=4)
    compare_segments(fw, ofw, "plus strand")
    compare_segments(rc, orc, "minus strand")
    assert st["num_hits"] == ost["num_hits"]
    assert len(fw) + len(rc) > 200


@pytest.mark.parametrize("xdrop,step", [(300, 16), (699, 16), (700, 16), (699, 8), (700, 8), (699, 32), (700, 32)])
def test_xdrop_scoring_forms(setup, xdrop, step):
    """With HOXD70 (largest score 100) an xdrop of at least 7 x 100 takes the
    lane kernel's windowed stop test, a smaller one its per-base test; both
    must reproduce the oracle, tile counts included."""
    w, sf = setup["w"], setup["sf"]
    p2 = oracle.params(xdrop=xdrop)
    sf.initialize_processor(False, CHUNK, 19, build_sub_mat(xdrop), xdrop, 3000, False)
    sf.set_tuning(step_bases=step)
    try:
        for rev in (False, True):
            text = setup["rctext"] if rev else w.query
            seeds = host_seeds(text, 0, CHUNK)
            got = sf.seed_and_filter(seeds, rev, 0)
            want, st = oracle.seed_and_filter(p2, setup["R"], setup["QR"] if rev else setup["Q"], setup["idx"],
                                              setup["pos"], seeds, rev)
            compare_segments(got, want, f"xdrop={xdrop} step={step} rev={rev}")
            assert sf.last_call_stats()["tiles"] == st["tiles_right"] + st["tiles_left"]
    finally:
        sf.set_tuning(step_bases=32)
        sf.initialize_processor(False, CHUNK, 19, build_sub_mat(910), 910, 3000, False)


@pytest.mark.parametrize("max_hits", [3000, 20000])
def test_max_hits_iterations(setup, max_hits):
    w, p, sf = setup["w"], setup["p"], setup["sf"]
    p2 = oracle.params(max_hits=max_hits)
    sf.set_max_hits(max_hits)
    try:
        seeds = host_seeds(w.query, 0, CHUNK)
        got = sf.seed_and_filter(seeds, False, 0)
        want, st = oracle.seed_and_filter(p2, setup["R"], setup["Q"], setup["idx"], setup["pos"], seeds, False)
        assert st["num_iter"] > 1
        assert sf.last_call_stats()["num_iter"] == st["num_iter"]
        compare_segments(got, want, f"MAX_HITS={max_hits}")
    finally:
        sf.set_max_hits(0)


@pytest.mark.parametrize("lane_cap,ctas,tile,step,sub", [(8, 2, 64, 8, 1), (16, 4, 1024, 16, 3), (32, 4, 1024, 8, 2),
                                                         (64, 3, 100, 16, 1), (512, 3, 1024, 8, 4), (4096, 3, 256, 16, 2),
                                                         (512, 2, 1024, 16, 8), (32, 3, 160, 32, 3), (4096, 2, 64, 32, 1),
                                                         (8192, 3, 160, 32, 4)])
def test_tuning_does_not_change_results(setup, lane_cap, ctas, tile, step, sub):
    """Every tuning gives the same HSPs and extends every hit exactly once (tile counts)."""
    w, p, sf = setup["w"], setup["p"], setup["sf"]
    seeds = host_seeds(w.query, 250_000, 500_000)
    want, st = oracle.seed_and_filter(p, setup["R"], setup["Q"], setup["idx"], setup["pos"], seeds, False)
    saved = sf.get_tuning()
    sf.set_tuning(lane_cap=lane_cap, ext_ctas_per_sm=ctas, tile_hits=tile, step_bases=step, substeps=sub)
    try:
        compare_segments(sf.seed_and_filter(seeds, False, 0), want,
                         f"lane_cap={lane_cap} ctas={ctas} step={step} substeps={sub}")
        assert sf.last_call_stats()["tiles"] == st["tiles_right"] + st["tiles_left"]
    finally:
        sf.set_tuning(**saved)


@pytest.mark.parametrize("sub,sw", [(1, 1), (2, 0), (2, 1), (3, 0), (3, 1), (8, 1)])
def test_switch_now_does_not_change_results(setup, sub, sw):
    """Starting a hit's left side in the same iteration as its right side ends
    (switch_now) or at the next one gives the same HSPs and tile counts."""
    w, p, sf = setup["w"], setup["p"], setup["sf"]
    for rev in (False, True):
        text = setup["rctext"] if rev else w.query
        seeds = host_seeds(text, 100_000, 300_000)
        want, st = oracle.seed_and_filter(p, setup["R"], setup["QR"] if rev else setup["Q"], setup["idx"],
                                          setup["pos"], seeds, rev)
        saved = sf.get_tuning()
        sf.set_tuning(substeps=sub, switch_now=sw)
        try:
            compare_segments(sf.seed_and_filter(seeds, rev, 0), want, f"substeps={sub} switch_now={sw} rev={rev}")
            assert sf.last_call_stats()["tiles"] == st["tiles_right"] + st["tiles_left"]
        finally:
            sf.set_tuning(**saved)


@pytest.mark.parametrize("lane_ctas,range_ctas", [(1, 1), (37, 16), (148, 148), (1000, 1024)])
def test_call_grid_knobs_do_not_change_results(setup, lane_ctas, range_ctas):
    """A plain call's lane-kernel grid and range-kernel grid (down to one CTA,
    and above the resident limit) give the same HSPs and tile counts."""
    w, p, sf = setup["w"], setup["p"], setup["sf"]
    seeds = host_seeds(w.query, 500_000, 700_000)
    want, st = oracle.seed_and_filter(p, setup["R"], setup["Q"], setup["idx"], setup["pos"], seeds, False)
    saved = sf.get_tuning()
    sf.set_tuning(call_lane_ctas=lane_ctas, call_range_ctas=range_ctas)
    try:
        compare_segments(sf.seed_and_filter(seeds, False, 0), want, f"call_lane_ctas={lane_ctas}")
        assert sf.last_call_stats()["tiles"] == st["tiles_right"] + st["tiles_left"]
    finally:
        sf.set_tuning(**saved)


def test_host_table_upload(setup):
    w, p, sf = setup["w"], setup["p"], setup["sf"]
    sf.send_seed_pos_table(setup["idx"], setup["pos"])
    seeds = host_seeds(w.query, 0, CHUNK)
    want, _ = oracle.seed_and_filter(p, setup["R"], setup["Q"], setup["idx"], setup["pos"], seeds, False)
    compare_segments(sf.seed_and_filter(seeds, False, 0), want, "host table")
    sf.generate_seed_pos_table(None, 1, 19, 12)


def test_transitions_small(built):
    rng = np.random.default_rng(7)
    T = random_text(rng, 200_000, lower=0.01)
    Q = bytearray(random_text(rng, 200_000))
    Q[50_000:60_000] = T[100_000:110_000]
    Q = bytes(Q)
    p = oracle.params(transition=True)
    idx, pos = oracle.build_table(T, p)
    sf = SeedFilter()
    sf.initialize_interface(1)
    sf.generate_shape_pos("12of19")
    sf.initialize_processor(True, 50_000, 19, build_sub_mat(910), 910, 3000, False)
    sf.send_ref_write_request(T)
    sf.generate_seed_pos_table(None, 1, 19, 12)
    sf.send_query_write_request(Q, 1)
    R, QC = oracle.encode(T), oracle.encode(Q)
    for j0 in range(0, len(Q) - 19, 50_000):
        seeds = host_seeds(Q, j0, min(j0 + 50_000, len(Q) - 19), transition=True)
        assert np.array_equal(seeds, oracle.chunk_seeds(Q, j0, min(j0 + 50_000, len(Q) - 19), p))
        got = sf.seed_and_filter(seeds, False, 1)
        want, _ = oracle.seed_and_filter(p, R, QC, idx, pos, seeds, False)
        compare_segments(got, want, f"transition chunk {j0}")
    # batched units (13 seed slots per position, device seeding) equal the per-call results, both strands
    QR = host_revcomp(Q)
    units, plain = [], []
    for rev, text in ((0, Q), (1, QR)):
        for j0 in range(0, len(Q) - 19, 50_000):
            j1 = min(j0 + 50_000, len(Q) - 19)
            units.append((1, rev, j0, j1))
            plain.append(sf.seed_and_filter(host_seeds(text, j0, j1, transition=True), bool(rev), 1))
    for u, (g, x) in enumerate(zip(sf.seed_and_filter_batch(units), plain)):
        compare_segments(g, x, f"batched transition unit {units[u]}")


@pytest.mark.parametrize("exclude,rm_knobs", [(False, None), (True, None), (True, (37, 3, 1)), (False, (600, 1, 1))])
def test_repeat_masker_self_alignment(built, exclude, rm_knobs):
    """rm calls against the oracle, with the default lane settings of an rm
    call and with other (rm_lane_ctas, rm_substeps, rm_switch_now)."""
    w = small_workload(scale=0.5, seed=9)
    T = w.target
    p = oracle.params(rm_exclude_diag=exclude)
    idx, pos = oracle.build_table(T, p)
    sf = SeedFilter()
    sf.initialize_interface(1)
    sf.generate_shape_pos("12of19")
    sf.initialize_processor(False, CHUNK, 19, build_sub_mat(910), 910, 3000, False)
    sf.send_ref_write_request(T)
    sf.generate_seed_pos_table(None, 1, 19, 12)
    sf.rm_send_query_write_request()
    sf.set_rm_exclude_diagonal(exclude)
    saved = sf.get_tuning()
    if rm_knobs:
        sf.set_tuning(rm_lane_ctas=rm_knobs[0], rm_substeps=rm_knobs[1], rm_switch_now=rm_knobs[2])
    try:
        R = oracle.encode(T)
        RC = oracle.rc_codes(R)
        rctext = host_revcomp(T)
        L = len(T)
        ref_start, ref_end = 50_000, 400_000
        for rev in (False, True):
            text = rctext if rev else T
            seeds = host_seeds(text, 100_000, 300_000)
            got = sf.rm_seed_and_filter(seeds, rev, ref_start, ref_end)
            want, st = oracle.seed_and_filter(p, R, RC if rev else R, idx, pos, seeds, rev, 1, ref_start, ref_end)
            assert st["hits_extended"] < st["num_hits"]
            compare_segments(got, want, f"rm rev={rev} exclude={exclude} knobs={rm_knobs}")
            assert sf.last_call_stats()["tiles"] == st["tiles_right"] + st["tiles_left"]
    finally:
        sf.set_rm_exclude_diagonal(False)
        sf.set_tuning(**saved)


def test_hsp_set_reused_after_overflow(setup):
    """The HSP set is emptied by each call's compaction and cleared in full
    only after a call that left it dirty: a call with more distinct HSPs than
    the workspace holds fails with SA_ERR_CAPACITY, and the next call on the
    same workspace still matches the oracle."""
    import os
    from segalign_b200 import SegAlignError
    w, p, sf = setup["w"], setup["p"], setup["sf"]
    seeds = host_seeds(w.query, 0, CHUNK)
    want_big, _ = oracle.seed_and_filter(p, setup["R"], setup["Q"], setup["idx"], setup["pos"], seeds, False)
    cap = 16
    assert len(want_big) - 1 > cap
    small = seeds[:4000]
    want_small, _ = oracle.seed_and_filter(p, setup["R"], setup["Q"], setup["idx"], setup["pos"], small, False)
    assert 0 < len(want_small) - 1 <= cap
    saved = {k: os.environ.get(k) for k in ("SA_SURV_CAP", "SA_SLOTS_PER_GPU")}
    os.environ["SA_SURV_CAP"] = str(cap)
    os.environ["SA_SLOTS_PER_GPU"] = "1"
    try:
        sf.generate_shape_pos("12of19")
        sf.initialize_processor(False, CHUNK, 19, build_sub_mat(910), 910, 3000, False)
        sf.send_ref_write_request(w.target)
        sf.generate_seed_pos_table(None, 1, 19, 12)
        sf.send_query_write_request(w.query, 0)
        compare_segments(sf.seed_and_filter(small, False, 0), want_small, "before overflow")
        with pytest.raises(SegAlignError) as ei:
            sf.seed_and_filter(seeds, False, 0)
        assert ei.value.code == -8  # SA_ERR_CAPACITY
        for _ in range(2):
            compare_segments(sf.seed_and_filter(small, False, 0), want_small, "after overflow")
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
        sf.initialize_processor(False, CHUNK, 19, build_sub_mat(910), 910, 3000, False)


def test_transitions_repeat_rich_sample(built):
    """The 600 Mbp workload's generator at 1% (6 Mbp target, GC 41%, 45%
    repeats, Alu-like families) with transitions on: eight 100 kbp units, both
    strands, GPU per call == oracle, header included."""
    w = synth.make(4, seed=104, scale=0.01)
    T, Q = w.target, w.query
    p = oracle.params(transition=True)
    idx, pos = oracle.build_table(T, p)
    sf = SeedFilter()
    sf.initialize_interface(1)
    sf.generate_shape_pos("12of19")
    sf.initialize_processor(True, 100_000, 19, build_sub_mat(910), 910, 3000, False)
    sf.send_ref_write_request(T)
    sf.generate_seed_pos_table(None, 1, 19, 12)
    sf.send_query_write_request(Q, 0)
    R, QF, QRC = oracle.encode(T), oracle.encode(Q), oracle.encode_rc(Q)
    QR = host_revcomp(Q)
    hits = hsps = 0
    for rev, text in ((0, Q), (1, QR)):
        for j0 in (0, 1_500_000, 3_000_000, 5_800_000):
            j1 = min(j0 + 100_000, len(Q) - 19)
            seeds = host_seeds(text, j0, j1, transition=True)
            got = sf.seed_and_filter(seeds, bool(rev), 0)
            want, st = oracle.seed_and_filter(p, R, QRC if rev else QF, idx, pos, seeds, bool(rev))
            compare_segments(got, want, f"repeat-rich transition unit rev={rev} [{j0},{j1})")
            hits += st["num_hits"]
            hsps += len(want) - 1
    assert hits > 5_000_000 and hsps > 50_000

