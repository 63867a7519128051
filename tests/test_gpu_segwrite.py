"""The segment writer on the GPU (sa_format_segments_gpu) writes the same
text, byte for byte, as the host writer, which the CPU tests pin to the
oracle's restatement of src/segment_printer.cpp:51-147."""
import numpy as np
import pytest

import oracle
import segalign_b200 as sa

pytestmark = pytest.mark.gpu


def _chroms(rng, n, prefix):
    chroms, at = [], 0
    for i in range(n):
        ln = int(rng.integers(1_000, 50_000))
        name = f"{prefix}{i + 1}" + ("_random_scaffold_with_a_long_name" if i % 3 == 2 else "")
        chroms.append((name, at, ln))
        at += ln + 1  # '&' separator
    return chroms, at - 1


def _case(seed, n_fw, n_rc):
    rng = np.random.default_rng(seed)
    ref, rlen = _chroms(rng, 7, "chr")
    query, _ = _chroms(rng, 9, "scaf")
    qb0 = query[3][1]
    qblen = query[7][1] + query[7][2] - qb0
    rb0 = ref[1][1]

    def hsps(n):
        a = np.zeros(n, dtype=sa.SEGMENT_DTYPE)
        a["ref_start"] = rng.integers(0, rlen - rb0 - 400, n)
        a["query_start"] = rng.integers(0, qblen - 400, n)
        a["len"] = rng.integers(0, 300, n)
        a["score"] = rng.integers(-50, 2_000_000, n)
        return a

    return ref, rb0, query, qb0, qblen, hsps(n_fw), hsps(n_rc)


@pytest.mark.parametrize("seed,n_fw,n_rc", [(1, 300, 200), (2, 0, 57), (3, 41, 0), (4, 0, 0), (5, 250_000, 180_000)])
def test_gpu_writer_equals_host_writer(built, seed, n_fw, n_rc):
    ref, rb0, query, qb0, qblen, fw, rc = _case(seed, n_fw, n_rc)
    host = sa.format_segments(ref, rb0, query, qb0, qblen, fw, rc)
    dev = sa.format_segments(ref, rb0, query, qb0, qblen, fw, rc, gpu=True)
    assert dev == host
    assert dev[0].count("\n") == n_fw and dev[1].count("\n") == n_rc


def test_gpu_writer_equals_oracle(built):
    ref, rb0, query, qb0, qblen, fw, rc = _case(6, 500, 400)
    fw["score"] = np.abs(fw["score"])
    rc["score"] = np.abs(rc["score"])
    assert sa.format_segments(ref, rb0, query, qb0, qblen, fw, rc, gpu=True) == \
        oracle.format_segments(ref, rb0, query, qb0, qblen, fw, rc)
