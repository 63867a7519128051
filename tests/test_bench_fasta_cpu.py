"""The whole-file leg of bench.py on CPU: the FASTA files it writes hold the
workload exactly (the target's '&'-joined chromosomes as one record each, the
query as its records), it passes the bench's interval, overlap and chunk sizes
to the whole-file driver, and it reports the driver's figures with the check
against the e2e leg.  The driver itself is replaced by a fake that reads the
files back; the GPU run of sa_align_fasta is covered by tests/test_ingest.py."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import bench  # noqa: E402
import oracle  # noqa: E402
from segalign_b200 import synth  # noqa: E402


class _FakeDriver:
    """Stands in for SeedFilter.align_fasta: parses the files with the
    oracle's restatement of the reader and records what it was given."""

    def __init__(self):
        self.kw = None
        self.target = self.query = None

    def align_fasta(self, target_path, query_path, **kw):
        self.kw = kw
        self.target = oracle.fasta_blocks(open(target_path, "rb").read(), 500_000_000)
        self.query = oracle.fasta_blocks(open(query_path, "rb").read(), 500_000_000)
        with open(kw["segments_path"], "wb") as f:
            f.write(b"segments")
        return dict(read_seconds=0.5, table_seconds=0.1, query_write_seconds=0.05, calls_seconds=0.3,
                    output_seconds=0.2, num_hits=1234, num_hsps=56)


def test_fasta_leg_writes_the_workload_and_reports_the_driver(built):
    w = synth.make(2, seed=102, scale=0.005)
    w = synth.Workload(w.target, w.query, w.target_chr, [(0, len(w.query))])
    drv = _FakeDriver()
    res = bench.run_fasta(drv, w, {"num_hits": 1234, "num_hsps": 56})
    text, chroms, blocks = drv.target  # one block; the text keeps the closing '&' outside the block length
    assert blocks == [(0, len(w.target))] and text[:len(w.target)] == w.target
    assert [(c[1], c[2]) for c in chroms] == [tuple(c) for c in w.target_chr]
    qtext, qchroms, qblocks = drv.query
    assert qblocks == [(0, len(w.query))] and qtext[:len(w.query)] == w.query and len(qchroms) == 1
    assert drv.kw["interval_size"] == bench.INTERVAL and drv.kw["interval_overlap"] == bench.OVERLAP
    assert drv.kw["chunk_size"] == bench.CHUNK
    assert res["hits"] == 1234 and res["hsps"] == 56 and res["same_hits_and_hsps_as_e2e"]
    assert res["segments_bytes"] == len(b"segments") and res["fasta_bytes"] > len(w.target) + len(w.query)
    assert res["extensions_per_s"] == 1234 / res["seconds"]
    assert not os.path.exists(os.path.dirname(drv.kw["segments_path"]))  # the leg cleans up its files
    # a run whose counts differ from the e2e leg's says so
    assert not bench.run_fasta(_FakeDriver(), w, {"num_hits": 1, "num_hsps": 56})["same_hits_and_hsps_as_e2e"]
