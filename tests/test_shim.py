"""The drop-in shim (include/segalign_b200_shim.hpp) with the reference's own
host code: tests/shim/Makefile compiles the glue file INTEGRATION.md shows
against the reference's headers (src/seed_filter.h, src/graph.h, src/store.h,
common/seed_filter_interface.h, common/ntcoding.h) and links the reference's
unchanged src/seeder.cpp, common/ntcoding.cpp and common/DRAM.cpp with
libsegalign_b200.so.  The GPU test runs that seeder over the 1 Mbp x 1 Mbp
workload through g_SeedAndFilter and compares both strands with the oracle's
restatement of the seeder pipeline, bit for bit."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import oracle
from tests.helpers import compare_segments, small_workload

HERE = os.path.dirname(os.path.abspath(__file__))
EXE = os.path.join(HERE, "shim", "_build", "shim_seeder")
REF_DIR = os.environ.get("SA_REFERENCE_DIR", "/root/reference")
HAVE_REF = os.path.isfile(os.path.join(REF_DIR, "src", "seeder.cpp"))


@pytest.mark.skipif(not HAVE_REF, reason="reference tree absent: the shim is compiled against its headers")
def test_shim_compiles_and_links_with_the_reference_seeder(built):
    r = subprocess.run(["make", "-s", "-C", os.path.join(HERE, "shim"), f"REF_DIR={REF_DIR}"], capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stderr
    syms = subprocess.run(["nm", "-C", EXE], capture_output=True, text=True).stdout
    for s in ("g_InitializeInterface", "g_SendRefWriteRequest", "g_ClearRef", "g_InitializeProcessor",
              "g_SendQueryWriteRequest", "g_SeedAndFilter", "g_ClearQuery", "g_ShutdownProcessor",
              "GenerateSeedPosTable", "SendSeedPosTable", "seeder_body::operator()"):
        assert s in syms, s
    libs = subprocess.run(["ldd", EXE], capture_output=True, text=True).stdout
    assert "libsegalign_b200.so" in libs


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(EXE), reason="shim seeder not built (needs the reference tree)")
def test_reference_seeder_through_shim_matches_oracle(built):
    w = small_workload()
    with tempfile.TemporaryDirectory() as d:
        t, q, o = (os.path.join(d, x) for x in ("t.txt", "q.txt", "o.bin"))
        open(t, "wb").write(w.target)
        open(q, "wb").write(w.query)
        r = subprocess.run([EXE, t, q, o], capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        raw = open(o, "rb").read()
    nf, nr, hits, seeds = np.frombuffer(raw[:32], dtype=np.uint64)
    recs = np.frombuffer(raw[32:], dtype=oracle.SEGMENT_DTYPE)
    fw, rc = recs[:nf], recs[nf:nf + nr]
    p = oracle.params()
    idx, pos = oracle.build_table(w.target, p)
    ofw, orc, st = oracle.pipeline(p, w.target, w.query, idx, pos, nthreads=4)
    compare_segments(fw, ofw, "plus strand through the shim")
    compare_segments(rc, orc, "minus strand through the shim")
    assert int(hits) == st["num_hits"]
    assert len(fw) + len(rc) > 200
