"""FASTA ingest, sequence blocks and the whole-file driver with double-buffered
query blocks (src/main.cpp:297-730).

CPU: sa_fasta_load joins records into '&'-separated blocks exactly as the
oracle's restatement of kseq's reading rules and src/main.cpp's block rules
does (multi-line records, empty lines, CRLF, comments, gzip, several block
sizes).  GPU: a multi-record target and query, each cut into two blocks, go
through sa_align_fasta; per target block, query block and strand its HSP lists
equal the oracle seeder pipeline on the same block texts, and its segments file
equals the oracle's segment writer interval by interval."""
import gzip
import os
import struct

import numpy as np
import pytest

import oracle
from segalign_b200 import SeedFilter, build_sub_mat, fasta_load, synth
from tests.helpers import compare_segments


def _fasta(records, rng, crlf=False, width=60):
    nl = "\r\n" if crlf else "\n"
    out = []
    for name, seq in records:
        out.append(f">{name} some comment{nl}")
        s = seq.decode()
        w = int(rng.integers(20, width + 1))
        for i in range(0, len(s), w):
            out.append(s[i:i + w] + nl)
            if rng.random() < 0.05:
                out.append(nl)  # empty line inside the record
    return "".join(out).encode()


def _records(rng, n, lo, hi):
    alph = np.frombuffer(b"ACGTacgtN", dtype=np.uint8)
    p = np.array([0.28, 0.18, 0.18, 0.28, 0.02, 0.02, 0.02, 0.01, 0.01])
    return [(f"chr{k}", rng.choice(alph, size=int(rng.integers(lo, hi)), p=p / p.sum()).tobytes()) for k in range(n)]


@pytest.mark.parametrize("crlf,gz", [(False, False), (True, False), (False, True)])
def test_fasta_blocks_match_restatement(built, tmp_path, crlf, gz):
    rng = np.random.default_rng(5 + crlf + 2 * gz)
    recs = _records(rng, 9, 1, 3000)
    data = _fasta(recs, rng, crlf=crlf)
    path = tmp_path / ("x.fa.gz" if gz else "x.fa")
    path.write_bytes(gzip.compress(data) if gz else data)
    for bs in (1, 500, 2500, 7000, 500_000_000):
        got = fasta_load(str(path), bs)
        text, chroms, blocks = oracle.fasta_blocks(data, bs)
        assert got["text"] == text, bs
        assert got["chroms"] == chroms, bs
        assert got["blocks"] == blocks, bs
    assert [c[0] for c in got["chroms"]] == [r[0] for r in recs]
    assert [c[2] for c in got["chroms"]] == [len(r[1]) for r in recs]


def _read_hsps(path):
    raw = open(path, "rb").read()
    n = len(raw) // 32
    a = np.frombuffer(raw, dtype=np.uint8).reshape(n, 32)
    keys = a[:, :16].copy().view(np.uint32).reshape(n, 4)
    recs = a[:, 16:].copy().reshape(-1).view(oracle.SEGMENT_DTYPE)
    return keys, recs


@pytest.mark.parametrize("crlf,gz", [(False, False), (True, False), (True, True)])
def test_fasta_long_lines_across_read_buffers(built, tmp_path, crlf, gz):
    """Lines of one base up to 1.5 Mbp, so that lines (and their CRLF pairs)
    start, end and break at many offsets of the reader's 1 MiB buffers, which
    it appends a span at a time; empty lines and records of one line.  Blocks
    equal the restatement's."""
    rng = np.random.default_rng(17 + crlf + 2 * gz)
    nl = b"\r\n" if crlf else b"\n"
    alph = np.frombuffer(b"ACGTacgtN", dtype=np.uint8)
    out = []
    for k in range(9):
        out.append(b">r%d comment" % k + nl)
        for _ in range(int(rng.integers(1, 6))):
            n = int(rng.choice([1, 2, int(rng.integers(3, 5000)), int(rng.integers(200_000, 1_500_000))]))
            out.append(rng.choice(alph, size=n).tobytes() + nl)
            if rng.random() < 0.3:
                out.append(nl)
    data = b"".join(out)
    assert len(data) > 2 * (1 << 20)
    path = tmp_path / ("long.fa.gz" if gz else "long.fa")
    path.write_bytes(gzip.compress(data, compresslevel=1) if gz else data)
    for bs in (1_000_000, 500_000_000):
        got = fasta_load(str(path), bs)
        text, chroms, blocks = oracle.fasta_blocks(data, bs)
        assert got["text"] == text, bs
        assert got["chroms"] == chroms, bs
        assert got["blocks"] == blocks, bs


def test_fastq_records_known_answers(built, tmp_path):
    """kseq's FASTQ rules, worked out by hand: a '+' line ends the sequence,
    quality lines are read until they are as long as it, and a record whose
    quality runs out first ends the input without being kept; records are
    joined with '&' as FASTA records are."""
    data = b"@r1 c\nACG\nT\n+\nII\nII\n@r2\nGG\n+r2\nII\n>r3\nTTA\n@r4\nACGTACGT\n+\nIII\n"
    path = tmp_path / "x.fq"
    path.write_bytes(data)
    got = fasta_load(str(path), 500_000_000)
    assert got["text"][:got["blocks"][0][1]] == b"ACGT&GG&TTA"
    assert got["chroms"] == [("r1", 0, 4), ("r2", 5, 2), ("r3", 8, 3)]
    assert got["blocks"] == [(0, 11)]


@pytest.mark.gpu
def test_align_fasta_two_blocks_matches_oracle(built, tmp_path):
    rng = np.random.default_rng(11)
    w = synth.make(1, seed=303, scale=0.6)  # 600 kbp target and query with homologous segments
    cut = lambda s, k: [s[i * len(s) // k:(i + 1) * len(s) // k] for i in range(k)]  # noqa: E731
    trecs = [(f"t{k}", x) for k, x in enumerate(cut(w.target, 3))]
    qrecs = [(f"q{k}", x) for k, x in enumerate(cut(w.query, 4))]
    tdata, qdata = _fasta(trecs, rng), _fasta(qrecs, rng)
    tp, qp = tmp_path / "t.fa", tmp_path / "q.fa.gz"
    tp.write_bytes(tdata)
    qp.write_bytes(gzip.compress(qdata))
    BS, IV, CH = 250_000, 120_000, 50_000  # blocks of ~2 records, several intervals and chunks each
    T, tch, tbl = oracle.fasta_blocks(tdata, BS)
    Q, qch, qbl = oracle.fasta_blocks(qdata, BS)
    assert len(tbl) == 2 and len(qbl) == 2

    sf = SeedFilter()
    sf.initialize_interface(1)
    sf.generate_shape_pos("12of19")
    sf.initialize_processor(False, CH, 19, build_sub_mat(910), 910, 3000, False)
    seg_path, hsp_path = tmp_path / "out.segments", tmp_path / "out.hsp"
    st = sf.align_fasta(str(tp), str(qp), str(seg_path), str(hsp_path), seq_block_size=BS, interval_size=IV,
                        chunk_size=CH, num_threads=4)
    assert st["ref_blocks"] == 2 and st["query_blocks"] == 2
    keys, recs = _read_hsps(hsp_path)

    p = oracle.params()
    want_seg = []
    total = 0
    for rb, (rs, rl) in enumerate(tbl):
        rtext = T[rs:rs + rl]
        idx, pos = oracle.build_table(rtext, p)
        for qb, (qs, ql) in enumerate(qbl):
            qtext = Q[qs:qs + ql]
            ofw, orc, _ = oracle.pipeline(p, rtext, qtext, idx, pos, nthreads=4, interval_size=IV, chunk_size=CH)
            sel = (keys[:, 0] == rb) & (keys[:, 1] == qb)
            compare_segments(recs[sel & (keys[:, 3] == 0)], ofw, f"target block {rb} query block {qb} plus")
            compare_segments(recs[sel & (keys[:, 3] == 1)], orc, f"target block {rb} query block {qb} minus")
            total += len(ofw) + len(orc)
            for iv in sorted(set(keys[sel, 2].tolist())):
                m = sel & (keys[:, 2] == iv)
                f, r = oracle.format_segments(tch, rs, qch, qs, ql, recs[m & (keys[:, 3] == 0)],
                                              recs[m & (keys[:, 3] == 1)])
                want_seg.append(f + r)
    assert total > 50
    assert seg_path.read_text() == "".join(want_seg)
    assert st["num_hsps"] == len(recs)
