"""The no-allocation SeedAndFilter entry point against the regular one.

sa_seed_and_filter_noalloc() is for callers that cannot let the library
allocate device memory during their run (a host program that owns all device
memory through its own fixed-budget pool, or a latency-bound loop that cannot
take the device-wide synchronisation of cudaMalloc/cudaFree).  Its scratch is
one fixed device array, so it also has to give the same answer on consecutive
calls that reuse that array.  This file is collected last on purpose.
"""
import numpy as np
import pytest

from segalign_b200 import SeedFilter, SegAlignError, build_sub_mat, host_revcomp, host_seeds
from tests.helpers import compare_segments, small_workload

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sf(built):
    w = small_workload()
    f = SeedFilter()
    f.initialize_interface(1)
    f.generate_shape_pos("12of19")
    f.initialize_processor(False, 250_000, 19, build_sub_mat(910), 910, 3000, False)
    f.send_ref_write_request(w.target)
    f.generate_seed_pos_table(None, 1, 19, 12)
    f.send_query_write_request(w.query, 0)
    f.w = w
    return f


def test_noalloc_matches_regular_entry_on_consecutive_calls(sf):
    q = sf.w.query
    rc = host_revcomp(q)
    calls = [(q, 0, 0, 250_000), (rc, 1, 250_000, 500_000), (q, 0, 500_000, 750_000)]
    for text, rev, a, b in calls:  # consecutive calls reuse the same scratch array
        seeds = host_seeds(text, a, b)
        want = sf.seed_and_filter(seeds, bool(rev), 0)
        got = sf.seed_and_filter_noalloc(seeds, bool(rev), 0)
        compare_segments(got, want, f"noalloc rev={rev} [{a},{b})")
        assert len(want) > 1


def test_noalloc_rejects_oversized_calls(sf):
    seeds = host_seeds(sf.w.query, 0, 250_000)
    small = np.zeros(1, dtype=[("ref_start", "<u4"), ("query_start", "<u4"), ("len", "<u4"), ("score", "<i4")])
    with pytest.raises(SegAlignError) as e:
        sf.seed_and_filter_noalloc(seeds, False, 0, out=small)
    assert e.value.code == -8  # SA_ERR_CAPACITY: output buffer too small
    # the regular path still agrees afterwards
    compare_segments(sf.seed_and_filter_noalloc(seeds, False, 0), sf.seed_and_filter(seeds, False, 0), "after reject")


def test_noalloc_rejects_more_seeds_than_its_limit(sf):
    # a processor whose MAX_SEEDS (300,000) is above the no-allocation limit (262,144)
    sf.initialize_processor(False, 300_000, 19, build_sub_mat(910), 910, 3000, False)
    seeds = (np.arange(270_000, dtype=np.uint64) % 1000) << np.uint64(32)
    with pytest.raises(SegAlignError) as e:
        sf.seed_and_filter_noalloc(seeds, False, 0)
    assert e.value.code == -8  # SA_ERR_CAPACITY, rejected before any device work
    sf.initialize_processor(False, 250_000, 19, build_sub_mat(910), 910, 3000, False)
    seeds = host_seeds(sf.w.query, 750_000, 999_000)
    compare_segments(sf.seed_and_filter_noalloc(seeds, False, 0), sf.seed_and_filter(seeds, False, 0), "re-init")


def test_noalloc_distinct_hsp_limit_then_next_call_recovers(built):
    """A call with more distinct HSPs than the shared array's HSP set holds
    (262,144) fails with SA_ERR_CAPACITY; it leaves the set dirty, and the next
    call through the same array must still equal the regular entry point."""
    from tests.helpers import random_text

    rng = np.random.default_rng(7)
    T = random_text(rng, 12_000_000)
    Q = random_text(rng, 300_000)
    f = SeedFilter()
    f.initialize_interface(1)
    f.generate_shape_pos("12of19")
    # hspthresh 300: almost every random hit is kept, each with its own HSP
    f.initialize_processor(False, 250_000, 19, build_sub_mat(910), 910, 300, False)
    f.send_ref_write_request(T)
    f.generate_seed_pos_table(None, 1, 19, 12)
    f.send_query_write_request(Q, 0)
    seeds = host_seeds(Q, 0, 250_000)
    want = f.seed_and_filter(seeds, False, 0)
    assert len(want) - 1 > 262_144
    big = np.zeros(len(want) + 16, dtype=want.dtype)  # room for the output: only the HSP set can overflow
    with pytest.raises(SegAlignError) as e:
        f.seed_and_filter_noalloc(seeds, False, 0, out=big)
    assert e.value.code == -8 and "distinct HSPs" in str(e.value)
    for a, b in ((0, 40_000), (100_000, 160_000)):
        s = host_seeds(Q, a, b)
        want = f.seed_and_filter(s, False, 0)
        got = f.seed_and_filter_noalloc(s, False, 0, out=np.zeros(len(want) + 16, dtype=want.dtype))
        compare_segments(got, want, f"after the overflow [{a},{b})")
