"""GPU edge cases of the C ABI against the oracle: calls with no seeds or no
hits, a query with no valid seed window, batched units with empty, single
and end-of-query windows, the MAX_SEEDS limit at and one past it, a seed key
outside the table, and a query identical to the target, so that every
extension runs into both sequence ends."""
import numpy as np
import pytest

import oracle
from segalign_b200 import SeedFilter, SegAlignError, build_sub_mat, host_revcomp, host_seeds
from tests.helpers import compare_segments, random_text

pytestmark = pytest.mark.gpu

CHUNK = 50_000


@pytest.fixture(scope="module")
def setup(built):
    rng = np.random.default_rng(21)
    T = random_text(rng, 300_000, lower=0.01, nfrac=0.001)
    Q = bytearray(random_text(rng, 200_000))
    Q[20_000:40_000] = T[100_000:120_000]  # a homologous block
    Q = bytes(Q)
    p = oracle.params()
    idx, pos = oracle.build_table(T, p)
    sf = SeedFilter()
    sf.initialize_interface(1)
    sf.generate_shape_pos("12of19")
    sf.initialize_processor(False, CHUNK, 19, build_sub_mat(910), 910, 3000, False)
    sf.send_ref_write_request(T)
    sf.generate_seed_pos_table(None, 1, 19, 12)
    sf.send_query_write_request(Q, 0)
    sf.send_query_write_request(b"N" * 100_000, 1)  # no valid seed window
    return dict(T=T, Q=Q, p=p, idx=idx, pos=pos, sf=sf, R=oracle.encode(T), QC=oracle.encode(Q),
                QR=oracle.encode_rc(Q))


def test_no_seeds_and_seeds_without_hits(setup):
    sf = setup["sf"]
    for rev in (False, True):
        out = sf.seed_and_filter(np.zeros(0, dtype=np.uint64), rev, 0)
        assert len(out) == 1 and tuple(out[0]) == (0, 0, 0, 0)
    idx = setup["idx"]
    empty = [k for k in range(1, 1 << 24, 9973) if idx[k] == idx[k - 1]][:64]
    assert len(empty) == 64
    seeds = np.array([(k << 32) | (1000 + i) for i, k in enumerate(empty)], dtype=np.uint64)
    out = sf.seed_and_filter(seeds, False, 0)
    want, st = oracle.seed_and_filter(setup["p"], setup["R"], setup["QC"], idx, setup["pos"], seeds, False)
    assert st["num_hits"] == 0
    compare_segments(out, want, "seeds without hits")


def test_query_without_valid_seed_windows(setup):
    sf = setup["sf"]
    assert len(host_seeds(b"N" * 100_000, 0, 100_000 - 19)) == 0
    outs = sf.seed_and_filter_batch([(1, 0, 0, 50_000), (1, 1, 10, 99_981)])
    for o in outs:
        assert len(o) == 1 and int(o[0]["len"]) == 0 and int(o[0]["score"]) == 0
    fw, rc, st = sf.seeder_run(b"N" * 100_000, buffer=1, strand=3, num_threads=2, chunk_size=CHUNK)
    assert len(fw) == 0 and len(rc) == 0 and st["num_hits"] == 0


def test_ragged_batched_windows(setup):
    """Empty, one-position and end-of-query windows of a batch equal the plain calls on them."""
    sf, Q = setup["sf"], setup["Q"]
    L = len(Q) - 19
    rct = host_revcomp(Q)
    units = [(0, 0, 500, 500), (0, 0, 25_000, 25_001), (0, 1, 0, 1), (0, 0, L - 1, L), (0, 1, L - 7, L),
             (0, 0, 20_000, 40_000), (0, 1, 160_000, 180_000), (0, 0, L - CHUNK, L)]
    outs = sf.seed_and_filter_batch(units)
    for (buf, rev, a, b), o in zip(units, outs):
        if a == b:
            assert len(o) == 1 and tuple(o[0]) == (0, 0, 0, 0)
            continue
        seeds = host_seeds(rct if rev else Q, a, b)
        want, _ = oracle.seed_and_filter(setup["p"], setup["R"], setup["QR"] if rev else setup["QC"], setup["idx"],
                                         setup["pos"], seeds, bool(rev))
        compare_segments(o, want, f"unit {(rev, a, b)}")


def test_max_seeds_limit_and_bad_keys(setup):
    sf = setup["sf"]
    seeds = host_seeds(setup["Q"], 0, len(setup["Q"]) - 19)[:CHUNK]
    assert len(seeds) == CHUNK  # exactly MAX_SEEDS (the WGA chunk)
    want, _ = oracle.seed_and_filter(setup["p"], setup["R"], setup["QC"], setup["idx"], setup["pos"], seeds, False)
    compare_segments(sf.seed_and_filter(seeds, False, 0), want, "MAX_SEEDS seeds")
    more = np.concatenate([seeds, seeds[:1]])
    with pytest.raises(SegAlignError) as ei:
        sf.seed_and_filter(more, False, 0)
    assert ei.value.code == -5  # SA_ERR_MAX_SEEDS
    bad = np.array([(np.uint64(1 << 24) << np.uint64(32)) | np.uint64(5)], dtype=np.uint64)
    with pytest.raises(SegAlignError) as ei:
        sf.seed_and_filter(bad, False, 0)
    assert ei.value.code == -6  # SA_ERR_BAD_SEED
    # the slot is still usable afterwards
    compare_segments(sf.seed_and_filter(seeds[:1000], False, 0),
                     oracle.seed_and_filter(setup["p"], setup["R"], setup["QC"], setup["idx"], setup["pos"],
                                            seeds[:1000], False)[0], "after errors")


def test_self_alignment_reaches_both_sequence_ends(built):
    """Query == target: the main-diagonal hits extend to position 0 and to
    the last base of both sequences (the edge path of the scan)."""
    rng = np.random.default_rng(4)
    T = random_text(rng, 120_000)
    p = oracle.params()
    idx, pos = oracle.build_table(T, p)
    sf = SeedFilter()
    sf.initialize_interface(1)
    sf.generate_shape_pos("12of19")
    sf.initialize_processor(False, CHUNK, 19, build_sub_mat(910), 910, 3000, False)
    sf.send_ref_write_request(T)
    sf.generate_seed_pos_table(None, 1, 19, 12)
    sf.send_query_write_request(T, 0)
    R = oracle.encode(T)
    for a, b in ((0, 200), (len(T) - 19 - 200, len(T) - 19)):
        seeds = host_seeds(T, a, b)
        got = sf.seed_and_filter(seeds, False, 0)
        want, _ = oracle.seed_and_filter(p, R, R, idx, pos, seeds, False)
        compare_segments(got, want, f"self {a}")
        full = [r for r in got[1:] if int(r["ref_start"]) == 0 and int(r["query_start"]) == 0]
        assert full and int(full[0]["len"]) == len(T) - 1
