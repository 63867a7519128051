"""C ABI surface and host-side logic, without a GPU.

- the CUDA library loads and exports every entry point declared in include/*.h;
- host C++ (scoring table, seeder words, reverse complement) matches the oracle;
- calls that need a device fail with a status code, never a CPU fallback.
"""
import ctypes as C
import os
import re

import numpy as np
import pytest

import oracle
import segalign_b200 as sa

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in ("segalign_b200.h", "segalign_b200_host.h"):
        txt = open(os.path.join(ROOT, "include", h)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names |= set(re.findall(r"\b(sa_[a-z0-9_]+)\s*\(", txt))
    return names


def test_library_exports_every_declared_symbol(built):
    lib = sa.load_library()
    names = declared_symbols()
    assert len(names) >= 25
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing
    assert set(sa.EXPORTS) == names


@pytest.mark.parametrize("amb", ["", "n", "iupac", "n,3,40", "x,3,40"])
@pytest.mark.parametrize("xdrop", [910, 500])
def test_sub_mat_matches_oracle(built, amb, xdrop):
    assert np.array_equal(sa.build_sub_mat(xdrop, amb), oracle.sub_mat(xdrop, amb))


def test_sub_mat_bad_ambiguous(built):
    with pytest.raises(sa.SegAlignError):
        sa.build_sub_mat(910, "n,x,3")


@pytest.mark.parametrize("shape", ["12of19", "14of22", "110100111"])
@pytest.mark.parametrize("transition", [False, True])
def test_host_seeder_matches_oracle(built, shape, transition):
    rng = np.random.default_rng(11)
    t = rng.choice(np.frombuffer(b"ACGTACGTACGTacgtN&", dtype=np.uint8), size=30000).tobytes()
    p = oracle.params(shape=shape, transition=transition)
    got = sa.host_seeds(t, 100, 29000 - p.seed_size, shape=shape, transition=transition)
    want = oracle.chunk_seeds(t, 100, 29000 - p.seed_size, p)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("size", [10000, 5_000_003])
def test_host_revcomp_matches_oracle(built, size):
    """Small inputs take one pass; inputs of 4 Mi characters or more are split
    into blocks on several threads (skipped characters shift the blocks)."""
    rng = np.random.default_rng(3)
    t = rng.choice(np.frombuffer(b"ACGTacgtNn&RY", dtype=np.uint8), size=size).tobytes()
    assert sa.host_revcomp(t) == oracle.revcomp_text(t)


def test_calls_without_device_fail_with_status(built):
    lib = sa.load_library()
    if os.path.exists("/dev/nvidia0"):
        pytest.skip("a GPU is present")
    assert lib.sa_initialize_interface(-1) == -9  # SA_ERR_NO_DEVICE
    # nothing is resident: every compute entry point refuses with a status
    ptr, n = C.POINTER(C.c_uint8)(), C.c_uint64()
    seeds = np.zeros(4, dtype=np.uint64)
    r = lib.sa_seed_and_filter(seeds.ctypes.data_as(C.POINTER(C.c_uint64)), 4, 0, 0, C.byref(ptr), C.byref(n))
    assert r == -2  # SA_ERR_STATE
    with pytest.raises(sa.SegAlignError):
        sa.SeedFilter().initialize_interface(-1)


def test_seeder_run_validates_arguments(built):
    lib = sa.load_library()
    cfg = sa.SeederCfg(10_000_000, 0, 0, 3, 1, 0, 0, 0)  # chunk_size 0
    fw, fl, rc, rl = C.POINTER(C.c_uint8)(), C.c_uint64(), C.POINTER(C.c_uint8)(), C.c_uint64()
    r = lib.sa_seeder_run(C.byref(cfg), b"ACGT" * 10, 40, C.byref(fw), C.byref(fl), C.byref(rc), C.byref(rl), None)
    assert r == -1


def test_tuning_validation(built):
    lib = sa.load_library()
    assert lib.sa_set_tuning(12, -1, -1, -1) == -1    # not a multiple of the step
    assert lib.sa_set_tuning_param(b"step_bases", 12) == -1
    assert lib.sa_set_tuning_param(b"no_such_knob", 1) == -1
    assert lib.sa_set_tuning(-1, 128, -1, -1) == -1   # the lane kernel is built for 256 threads
    assert lib.sa_set_tuning(64, 256, 4, 1024) == 0
    assert lib.sa_set_tuning(512, 256, 3, 1024) == 0
    assert lib.sa_set_tuning(-1, -1, -1, 2048) == -1  # shared-memory tiles hold at most 1024 hits
    assert lib.sa_get_tuning_param(b"tile_hits") == 1024
    assert lib.sa_set_tuning(8192, 256, 3, 160) == 0


def test_named_tuning_parameters(built):
    """Each named knob accepts its documented range, rejects values outside it
    without changing the current value, and reads back what was set."""
    lib = sa.load_library()
    ranges = {b"substeps": (1, 8), b"rm_substeps": (1, 8), b"switch_now": (0, 1), b"rm_switch_now": (0, 1),
              b"range_ctas": (1, 1024), b"call_range_ctas": (1, 1024), b"call_lane_ctas": (0, 8192),
              b"rm_lane_ctas": (0, 8192)}
    for name, (lo, hi) in ranges.items():
        old = lib.sa_get_tuning_param(name)
        assert lo <= old <= hi, (name, old)
        for bad in (lo - 1, hi + 1):
            assert lib.sa_set_tuning_param(name, bad) == -1, (name, bad)
            assert lib.sa_get_tuning_param(name) == old
        for good in (lo, hi, old):
            assert lib.sa_set_tuning_param(name, good) == 0, (name, good)
            assert lib.sa_get_tuning_param(name) == good
    assert lib.sa_get_tuning_param(b"no_such_knob") == -1


def test_serve_calls_without_a_running_loop(built):
    """Serving calls report SA_ERR_STATE until sa_serve_start succeeds; stop is harmless."""
    import ctypes as C
    lib = sa.load_library()
    rid = C.c_uint64()
    assert lib.sa_serve_submit(b"ACGTACGT", 8, C.byref(rid)) == -2
    fw, rc = C.POINTER(C.c_uint8)(), C.POINTER(C.c_uint8)()
    n1, n2 = C.c_uint64(), C.c_uint64()
    assert lib.sa_serve_wait(1, 0, C.byref(fw), C.byref(n1), C.byref(rc), C.byref(n2), None) == -2
    assert lib.sa_serve_stop() == 0
    if not os.path.exists("/dev/nvidia0"):
        assert lib.sa_serve_start(None) == -2  # no interface, target or table


def test_autotune_needs_a_processor(built):
    import ctypes as C
    lib = sa.load_library()
    if os.path.exists("/dev/nvidia0"):
        pytest.skip("a GPU is present")
    u = (sa.Unit * 1)(sa.Unit(0, 0, 0, 100))
    res = sa.AutotuneResult()
    assert lib.sa_autotune(u, 1, None, C.byref(res)) == -2  # SA_ERR_STATE
    assert lib.sa_autotune(None, 0, None, C.byref(res)) == -1


def _random_chroms(rng, n, first=0):
    chroms, at = [], first
    for i in range(n):
        ln = int(rng.integers(1_000, 50_000))
        chroms.append((f"chr{i + 1}", at, ln))
        at += ln + 1  # '&' separator
    return chroms, at - 1


def test_segment_writer_matches_oracle(built):
    """.segments lines (src/segment_printer.cpp:51-147) from the C++ writer
    equal the oracle's restatement, for a query block in the middle of a
    multi-chromosome query and HSPs spread over its chromosomes."""
    rng = np.random.default_rng(5)
    ref, rlen = _random_chroms(rng, 7)
    query, qlen = _random_chroms(rng, 9)
    qb0 = query[3][1]
    qblen = query[7][1] + query[7][2] - qb0
    rb0 = ref[1][1]

    def hsps(n):
        a = np.zeros(n, dtype=sa.SEGMENT_DTYPE)
        a["ref_start"] = rng.integers(0, rlen - rb0 - 400, n)
        a["query_start"] = rng.integers(0, qblen - 400, n)
        a["len"] = rng.integers(1, 300, n)
        a["score"] = rng.integers(3000, 20000, n)
        return a

    fw, rc = hsps(300), hsps(200)
    got = sa.format_segments(ref, rb0, query, qb0, qblen, fw, rc)
    want = oracle.format_segments(ref, rb0, query, qb0, qblen, fw, rc)
    assert got == want
    assert got[0].count("\n") == 300 and got[1].count("\n") == 200 and "\t-\t" in got[1]


def test_rm_interval_writer_matches_oracle(built):
    rng = np.random.default_rng(6)
    chroms, total = _random_chroms(rng, 5)
    runs = np.zeros(50, dtype=sa.RM_RUN_DTYPE)
    runs["query_start"] = np.sort(rng.integers(0, total - 600, 50))
    runs["len"] = rng.integers(1, 500, 50)
    for markend in (False, True):
        assert sa.format_rm_intervals(chroms, 0, runs, markend) == oracle.format_rm_intervals(chroms, 0, runs, markend)
    assert sa.format_rm_intervals(chroms, 0, runs[:0], True) == ""
