"""ctypes binding of the CPU oracle (oracle/sa_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline / reference legs as the checker or the timed CPU
baseline.  The product path (segalign_b200) never uses it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "build", "libsa_oracle.so")
REF_LIB_PATH = os.path.join(HERE, "_ref", "libref_ntcoding.so")
SEGMENT_DTYPE = np.dtype([("ref_start", "<u4"), ("query_start", "<u4"), ("len", "<u4"), ("score", "<i4")])
_P = C.POINTER


class Params(C.Structure):
    _fields_ = [("sub_mat", C.c_int32 * 64), ("xdrop", C.c_int32), ("hspthresh", C.c_int32),
                ("noentropy", C.c_int32), ("seed_size", C.c_int32), ("kmer_size", C.c_int32),
                ("shape_pos", C.c_int32 * 32), ("transition", C.c_int32), ("rm_exclude_diag", C.c_int32),
                ("max_hits", C.c_uint64)]


class Stats(C.Structure):
    _fields_ = [("num_seeds", C.c_uint64), ("num_hits", C.c_uint64), ("hits_extended", C.c_uint64),
                ("tiles_right", C.c_uint64), ("tiles_left", C.c_uint64), ("survivors", C.c_uint64),
                ("num_hsps", C.c_uint64), ("unpinned", C.c_uint64), ("base_steps", C.c_uint64),
                ("num_iter", C.c_int32), ("pad", C.c_int32)]


class HitResult(C.Structure):
    _fields_ = [("right_best", C.c_int32), ("right_pos", C.c_int32), ("left_best", C.c_int32),
                ("left_pos", C.c_int32), ("total", C.c_int32), ("keep", C.c_int32), ("score", C.c_int32),
                ("entropy_branch", C.c_int32), ("entropy", C.c_double), ("tiles_right", C.c_uint32),
                ("tiles_left", C.c_uint32), ("unpinned", C.c_int32), ("pad", C.c_int32)]


class PipelineCfg(C.Structure):
    _fields_ = [("interval_size", C.c_uint32), ("interval_overlap", C.c_uint32), ("chunk_size", C.c_uint32),
                ("strand", C.c_int32), ("nthreads", C.c_int32), ("max_chunks", C.c_uint32)]


_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        u8p, u32p, u64p = _P(C.c_uint8), _P(C.c_uint32), _P(C.c_uint64)
        segpp = _P(_P(C.c_uint8))
        sig = {
            "or_encode": (None, [C.c_char_p, C.c_uint64, u8p]),
            "or_encode_rc": (None, [C.c_char_p, C.c_uint64, u8p]),
            "or_rc_codes": (None, [u8p, C.c_uint64, u8p]),
            "or_revcomp_text": (C.c_uint64, [C.c_char_p, C.c_char_p, C.c_uint64]),
            "or_build_sub_mat": (C.c_int, [C.c_int, C.c_char_p, _P(C.c_int32)]),
            "or_parse_shape": (C.c_int, [C.c_char_p, _P(Params)]),
            "or_kmer_index": (C.c_uint32, [C.c_char_p, C.c_uint64, _P(Params)]),
            "or_table_count": (C.c_uint64, [C.c_char_p, C.c_uint32, C.c_uint32, _P(Params)]),
            "or_build_table": (C.c_int, [C.c_char_p, C.c_uint32, C.c_uint32, _P(Params), u32p, u32p, C.c_uint64, u64p]),
            "or_chunk_seeds": (C.c_uint64, [C.c_char_p, C.c_uint32, C.c_uint32, _P(Params), u64p, C.c_uint64]),
            "or_seed_and_filter": (C.c_int, [_P(Params), u8p, C.c_uint32, u8p, C.c_uint32, u32p, u32p, u64p,
                                             C.c_uint64, C.c_int, C.c_int, C.c_uint32, C.c_uint32, segpp, u64p,
                                             _P(Stats)]),
            "or_free": (None, [C.c_void_p]),
            "or_extend_hit": (None, [_P(Params), u8p, C.c_uint32, u8p, C.c_uint32, C.c_uint32, C.c_uint32,
                                     _P(HitResult)]),
            "or_pipeline": (C.c_int, [_P(Params), _P(PipelineCfg), C.c_char_p, C.c_uint32, C.c_char_p, C.c_uint32,
                                      u32p, u32p, segpp, u64p, segpp, u64p, _P(Stats)]),
            "or_rm_plan": (C.c_uint64, [C.c_uint64, C.c_uint32, C.c_uint32, C.c_float, C.c_uint32, u32p,
                                        C.c_uint64]),
            "or_rm_intervals": (C.c_uint64, [_P(SEGSTRUCT := C.c_uint8), C.c_uint64, C.c_uint32, C.c_uint32, u32p,
                                             u32p, C.c_uint64, u8p]),
        }
        for k, (r, a) in sig.items():
            f = getattr(L, k)
            f.restype = r
            f.argtypes = a
        _lib = L
    return _lib


def ref_ntcoding() -> C.CDLL | None:
    """The reference's own common/ntcoding.cpp (built by `make -C oracle ref`), or None."""
    if not os.path.exists(REF_LIB_PATH):
        return None
    L = C.CDLL(REF_LIB_PATH)
    L.ref_generate_shape_pos.restype = C.c_int
    L.ref_generate_shape_pos.argtypes = [C.c_char_p]
    L.ref_is_transition_at_pos.restype = C.c_int
    L.ref_is_transition_at_pos.argtypes = [C.c_int]
    L.ref_get_kmer_index_at_pos.restype = C.c_uint32
    L.ref_get_kmer_index_at_pos.argtypes = [C.c_char_p, C.c_size_t, C.c_uint32]
    L.ref_revcomp.restype = None
    L.ref_revcomp.argtypes = [C.c_char_p, C.c_char_p, C.c_size_t, C.c_size_t, C.c_size_t]
    return L


def params(xdrop=910, hspthresh=3000, noentropy=False, shape="12of19", transition=False, ambiguous="",
           max_hits=1 << 40, rm_exclude_diag=False) -> Params:
    p = Params()
    L = lib()
    if L.or_build_sub_mat(xdrop, ambiguous.encode(), p.sub_mat) != 0:
        raise ValueError("bad ambiguous")
    if L.or_parse_shape(shape.encode(), C.byref(p)) < 0:
        raise ValueError("bad shape")
    p.xdrop, p.hspthresh, p.noentropy = xdrop, hspthresh, int(noentropy)
    p.transition, p.max_hits, p.rm_exclude_diag = int(transition), max_hits, int(rm_exclude_diag)
    return p


def encode(text: bytes) -> np.ndarray:
    out = np.empty(len(text), dtype=np.uint8)
    lib().or_encode(text, len(text), out.ctypes.data_as(_P(C.c_uint8)))
    return out


def encode_rc(text: bytes) -> np.ndarray:
    out = np.empty(len(text), dtype=np.uint8)
    lib().or_encode_rc(text, len(text), out.ctypes.data_as(_P(C.c_uint8)))
    return out


def rc_codes(codes: np.ndarray) -> np.ndarray:
    c = np.ascontiguousarray(codes, dtype=np.uint8)
    out = np.empty_like(c)
    lib().or_rc_codes(c.ctypes.data_as(_P(C.c_uint8)), len(c), out.ctypes.data_as(_P(C.c_uint8)))
    return out


def revcomp_text(text: bytes) -> bytes:
    dst = C.create_string_buffer(len(text))
    n = lib().or_revcomp_text(dst, text, len(text))
    return dst.raw[:n]


def sub_mat(xdrop=910, ambiguous="") -> np.ndarray:
    m = (C.c_int32 * 64)()
    if lib().or_build_sub_mat(xdrop, ambiguous.encode(), m) != 0:
        raise ValueError("bad ambiguous")
    return np.array(list(m), dtype=np.int32)


def build_table(text: bytes, p: Params, step: int = 1):
    L = lib()
    n = L.or_table_count(text, len(text), step, C.byref(p))
    idx = np.zeros(1 << (2 * p.kmer_size), dtype=np.uint32)
    pos = np.zeros(max(n, 1), dtype=np.uint32)
    ni = C.c_uint64()
    r = L.or_build_table(text, len(text), step, C.byref(p), idx.ctypes.data_as(_P(C.c_uint32)),
                         pos.ctypes.data_as(_P(C.c_uint32)), len(pos), C.byref(ni))
    assert r == 0
    return idx, pos[: ni.value]


def chunk_seeds(text: bytes, j0: int, j1: int, p: Params) -> np.ndarray:
    L = lib()
    n = L.or_chunk_seeds(text, j0, j1, C.byref(p), None, 0)
    out = np.empty(max(n, 1), dtype=np.uint64)
    L.or_chunk_seeds(text, j0, j1, C.byref(p), out.ctypes.data_as(_P(C.c_uint64)), n)
    return out[:n]


def _segs(ptr, n):
    try:
        if n == 0:
            return np.zeros(0, dtype=SEGMENT_DTYPE)
        buf = C.cast(ptr, _P(C.c_uint8 * (16 * n))).contents
        return np.frombuffer(bytes(buf), dtype=SEGMENT_DTYPE).copy()
    finally:
        lib().or_free(ptr)


def seed_and_filter(p: Params, ref_codes: np.ndarray, query_codes: np.ndarray, index: np.ndarray, pos: np.ndarray,
                    seeds: np.ndarray, rev: bool, mode: int = 0, rm_ref_start: int = 0, rm_ref_end: int = 0):
    """Returns (segments with header, stats dict); raises on an oracle error code."""
    L = lib()
    s = np.ascontiguousarray(seeds, dtype=np.uint64)
    ptr, n, st = _P(C.c_uint8)(), C.c_uint64(), Stats()
    r = L.or_seed_and_filter(C.byref(p), ref_codes.ctypes.data_as(_P(C.c_uint8)), len(ref_codes),
                             query_codes.ctypes.data_as(_P(C.c_uint8)), len(query_codes),
                             index.ctypes.data_as(_P(C.c_uint32)), pos.ctypes.data_as(_P(C.c_uint32)),
                             s.ctypes.data_as(_P(C.c_uint64)), len(s), int(rev), mode, rm_ref_start, rm_ref_end,
                             C.byref(ptr), C.byref(n), C.byref(st))
    if r != 0:
        raise RuntimeError(f"oracle seed_and_filter error {r}")
    return _segs(ptr, n.value), {k: getattr(st, k) for k, _ in Stats._fields_ if k != "pad"}


def extend_hit(p: Params, ref_codes, query_codes, ref_loc: int, query_loc: int) -> dict:
    h = HitResult()
    lib().or_extend_hit(C.byref(p), ref_codes.ctypes.data_as(_P(C.c_uint8)), len(ref_codes),
                        query_codes.ctypes.data_as(_P(C.c_uint8)), len(query_codes), ref_loc, query_loc, C.byref(h))
    return {k: getattr(h, k) for k, _ in HitResult._fields_ if k != "pad"}


def pipeline(p: Params, ref_text: bytes, query_text: bytes, index, pos, strand=3, nthreads=1,
             interval_size=10_000_000, chunk_size=250_000, interval_overlap=0, max_chunks=0):
    """Seeder pipeline over one query block (src/seeder.cpp:47-121) -> (fw, rc, stats)."""
    L = lib()
    cfg = PipelineCfg(interval_size, interval_overlap, chunk_size, strand, nthreads, max_chunks)
    fw, fl, rc, rl, st = _P(C.c_uint8)(), C.c_uint64(), _P(C.c_uint8)(), C.c_uint64(), Stats()
    r = L.or_pipeline(C.byref(p), C.byref(cfg), ref_text, len(ref_text), query_text, len(query_text),
                      index.ctypes.data_as(_P(C.c_uint32)), pos.ctypes.data_as(_P(C.c_uint32)), C.byref(fw),
                      C.byref(fl), C.byref(rc), C.byref(rl), C.byref(st))
    if r != 0:
        raise RuntimeError(f"oracle pipeline error {r}")
    return _segs(fw, fl.value), _segs(rc, rl.value), {k: getattr(st, k) for k, _ in Stats._fields_ if k != "pad"}


def rm_intervals(hsps: np.ndarray, block_len: int, M: int):
    """repeat_masker_src/seeder.cpp:151-186 coverage runs -> (starts, lens)."""
    L = lib()
    h = np.ascontiguousarray(hsps, dtype=SEGMENT_DTYPE)
    cnt = np.zeros(block_len, dtype=np.uint8)
    n = L.or_rm_intervals(h.ctypes.data_as(_P(C.c_uint8)), len(h), block_len, M, None, None, 0,
                          cnt.ctypes.data_as(_P(C.c_uint8)))
    st = np.zeros(max(n, 1), dtype=np.uint32)
    ln = np.zeros(max(n, 1), dtype=np.uint32)
    L.or_rm_intervals(h.ctypes.data_as(_P(C.c_uint8)), len(h), block_len, M, st.ctypes.data_as(_P(C.c_uint32)),
                      ln.ctypes.data_as(_P(C.c_uint32)), n, cnt.ctypes.data_as(_P(C.c_uint8)))
    return st[:n], ln[:n]


def rm_plan(seq_len: int, interval_size: int, block_size: int, prop_neigh: float, seed_size: int = 19) -> np.ndarray:
    """repeat_masker_src/main.cpp:319-428 -> rows (block, block_start, block_len, start, end, ref_start, ref_end)."""
    L = lib()
    n = L.or_rm_plan(seq_len, interval_size, block_size, prop_neigh, seed_size, None, 0)
    out = np.zeros((max(n, 1), 7), dtype=np.uint32)
    L.or_rm_plan(seq_len, interval_size, block_size, prop_neigh, seed_size, out.ctypes.data_as(_P(C.c_uint32)), n)
    return out[:n]


def _chrom_index(starts, x):
    import bisect
    return max(bisect.bisect_right(starts, x) - 1, 0)


def format_segments(ref_chroms, r_block_start, q_chroms, q_block_start, q_block_len, fw, rc):
    """src/segment_printer.cpp:51-147 (the .segments lines; the lastz command
    lines are out of scope).  Chromosome tables: [(name, global start, len)].
    The reference caches the current query chromosome, which picks the same
    chromosome as its upper_bound lookup for every position inside one."""
    rstarts = [c[1] for c in ref_chroms]
    qstarts = [c[1] for c in q_chroms]
    block = [c for c in q_chroms if q_block_start <= c[1] < q_block_start + q_block_len]
    # src/main.cpp:355-362: rc table = the block's chromosomes in reverse order
    rct = [(n, 2 * q_block_start + q_block_len - st - ln, ln) for (n, st, ln) in reversed(block)]
    rcstarts = [c[1] for c in rct]

    def lines(hsps, table, starts, strand):
        out = []
        for e in hsps:
            sr = int(e["ref_start"]) + r_block_start
            rn, rs, _ = ref_chroms[_chrom_index(rstarts, sr)]
            sq = q_block_start + int(e["query_start"])
            qn, qs, _ = table[_chrom_index(starts, sq)]
            ln = int(e["len"])
            out.append(f"{rn}\t{sr + 1 - rs}\t{sr + ln + 1 - rs}\t{qn}\t{sq + 1 - qs}\t{sq + ln + 1 - qs}\t{strand}\t"
                       f"{int(e['score'])}\n")
        return "".join(out)

    return lines(fw, q_chroms, qstarts, "+"), lines(list(rc)[::-1], rct, rcstarts, "-")


def format_rm_intervals(chroms, block_start, runs, markend=False):
    """repeat_masker_src/segment_printer.cpp:24-62."""
    starts = [c[1] for c in chroms]
    out = []
    for r in runs:
        sq = block_start + int(r["query_start"])
        n, st, _ = chroms[_chrom_index(starts, sq)]
        out.append(f"{n}\t{sq - st}\t{sq + int(r['len']) + 1 - st}\n")
    if out and markend:
        out.append("# segalign_repeat_masker end-of-file\n")
    return "".join(out)


# --------------------------------------------------------------------------
# The reference's own seed-filter code on the GPU (oracle/ref_harness.cu,
# built by `make -C oracle ref_kernels` from the reference tree).  It pins the
# oracle's extension/dedup half; it needs a GPU, and its binaries travel with
# the repository snapshot (oracle/_ref/ is git-ignored, not copy-ignored).
# --------------------------------------------------------------------------
REF_HARNESS = {"plain": os.path.join(HERE, "_ref", "ref_seedfilter"),
               "rm": os.path.join(HERE, "_ref", "ref_seedfilter_rm")}

# src/main.cpp:152-171: named shapes in the T/0 form GenerateShapePos reads.
_T_SHAPES = {"12of19": "TTT0T00TT00T0T0TTTT", "14of22": "TTT0T0TT00TT00T0T0TTTT"}


def ref_harness_available(mode: str = "plain") -> bool:
    return os.path.exists(REF_HARNESS[mode])


def shape_t_form(shape: str) -> str:
    return _T_SHAPES.get(shape, shape.replace("1", "T"))


def ref_safe_texts(target: bytes, query: bytes) -> tuple[bytes, bytes]:
    """Inputs on which the reference's find_hsps never indexes its short[4]
    count arrays with a code >= 4 (src/seed_filter.cu:416-423,567-573): target
    N/n become lowercase 'a' and query lowercase becomes 'N'.  Seeds are
    unchanged (both classes invalidate a seed window, common/ntcoding.cpp:10-19)
    and so is every score (L and N score -1000 against every code, L-N included,
    src/main.cpp:180-261); only pairs of equal non-ACGT codes disappear."""
    t = np.frombuffer(target, dtype=np.uint8).copy()
    t[(t == ord("N")) | (t == ord("n"))] = ord("a")
    q = np.frombuffer(query, dtype=np.uint8).copy()
    q[(q >= ord("a")) & (q <= ord("z"))] = ord("N")
    return t.tobytes(), q.tobytes()


def ref_tail_keys(target: bytes, p: Params) -> np.ndarray:
    """Keys of the seed windows that start within 32 bases (+ seed size) of the
    target end; a hit on one of them would start a tile past the end."""
    L = len(target)
    ss = p.seed_size
    keys = [lib().or_kmer_index(target, q, C.byref(p)) for q in range(max(L - ss - 31, 0), L - ss + 1)]
    return np.array([k for k in keys if k != (1 << 31)], dtype=np.uint64)


def ref_filter_seeds(seeds: np.ndarray, tail_keys: np.ndarray, query_len: int, seed_size: int = 19) -> np.ndarray:
    """Drops seeds whose hits could start a tile past a sequence end (the
    harness refuses them; see oracle/ref_harness.cu)."""
    s = np.ascontiguousarray(seeds, dtype=np.uint64)
    keep = (s & np.uint64(0xFFFFFFFF)) + np.uint64(seed_size + 32) <= np.uint64(query_len)
    if len(tail_keys):
        keep &= ~np.isin(s >> np.uint64(32), tail_keys)
    return s[keep]


def ref_seed_and_filter(calls, target: bytes, query: bytes | None = None, *, mode: str = "plain", xdrop=910,
                        hspthresh=3000, noentropy=False, shape="12of19", transition=False, max_hits: int = 0,
                        wga_chunk: int = 250_000, step: int = 1, records: bool = True, ambiguous: str = "",
                        timeout: float = 1200, workdir: str | None = None) -> list[dict]:
    """Runs the reference's own SeedAndFilter (src/seed_filter.cu:654-778, or
    repeat_masker_src/seed_filter.cu:723-855 for mode "rm") over `calls` in one
    process, after its own InitializeInterface / SendRefWriteRequest /
    InitializeProcessor / GenerateSeedPosTable / SendQueryWriteRequest.

    Each call is a dict: `rev`; `seeds` (uint64 words) or `range` = (j0, j1)
    for seeds made by the harness as src/seeder.cpp:57-74; rm calls also give
    `ref_start`, `ref_end`.  Returns per call {"segments" (header row first,
    its ref_start/query_start zero), "num_seeds", "num_hits", "seconds"}."""
    import struct
    import tempfile

    exe = REF_HARNESS[mode]
    if not os.path.exists(exe):
        raise FileNotFoundError(f"{exe} missing: run `make -C oracle ref_kernels` where the reference tree is")
    sm = sub_mat(xdrop, ambiguous)
    ts = shape_t_form(shape).encode()
    q = b"" if mode == "rm" else (query or b"")
    with tempfile.TemporaryDirectory(dir=workdir) as d:
        fin, fout = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
        with open(fin, "wb") as f:
            f.write(b"SAREFIN1")
            f.write(struct.pack("<IIIiiIII", 1 if mode == "rm" else 0, int(transition), int(noentropy), xdrop,
                                hspthresh, wga_chunk, step, int(records)))
            f.write(struct.pack("<qI", int(max_hits), len(ts)) + ts)
            f.write(sm.astype("<i4").tobytes())
            f.write(struct.pack("<Q", len(target)) + target)
            f.write(struct.pack("<Q", len(q)) + q)
            f.write(struct.pack("<I", len(calls)))
            for c in calls:
                a, b = (c["ref_start"], c["ref_end"]) if mode == "rm" else (c.get("buffer", 0), 0)
                f.write(struct.pack("<III", int(c["rev"]), a, b))
                if "seeds" in c:
                    s = np.ascontiguousarray(c["seeds"], dtype="<u8")
                    f.write(struct.pack("<IQ", 0, len(s)) + s.tobytes())
                else:
                    f.write(struct.pack("<III", 1, *c["range"]))
        r = subprocess.run([exe, fin, fout], capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"reference harness exit {r.returncode}: {r.stderr.strip()[-2000:]}")
        out = []
        with open(fout, "rb") as f:
            assert f.read(8) == b"SAREFOUT"
            (n_calls,) = struct.unpack("<I", f.read(4))
            for _ in range(n_calls):
                n, ns, secs, hlen, hscore = struct.unpack("<QQdIi", f.read(32))
                segs = np.zeros(n, dtype=SEGMENT_DTYPE)
                segs[0]["len"], segs[0]["score"] = hlen, hscore
                if records and n > 1:
                    segs[1:] = np.frombuffer(f.read(16 * (n - 1)), dtype=SEGMENT_DTYPE)
                out.append({"segments": segs if records else segs[:1], "num_seeds": ns,
                            "num_hits": hscore & 0xFFFFFFFF, "num_hsps": hlen, "seconds": secs})
    return out


# --------------------------------------------------------------------------
# FASTA ingest and blocks (pure Python restatement; small inputs only)
# --------------------------------------------------------------------------
def fasta_records(data: bytes):
    """kseq's reading rules (common/kseq.h:183-224): records start at '>' or
    '@'; name = header up to the first white space; sequence lines follow
    until a line starting with '>', '+' or '@'; empty lines are skipped; a
    line's trailing '\\r' is dropped once the sequence is longer than one
    character.  FASTA only (no '+' quality sections)."""
    recs = []
    i, n = 0, len(data)
    pending = False
    while True:
        if not pending:
            while i < n and data[i] not in b">@":
                i += 1
            if i >= n:
                return recs
            i += 1
        pending = False
        j = i
        while j < n and not chr(data[j]).isspace():
            j += 1
        if j >= n and j == i:
            return recs
        name = data[i:j].decode()
        i = j
        if i < n and data[i] != ord("\n"):
            while i < n and data[i] != ord("\n"):
                i += 1
        i += 1  # past the header's newline (or the delimiter)
        seq = bytearray()
        while i < n and data[i] not in b">+@":
            if data[i] == ord("\n"):
                i += 1
                continue
            k = data.find(b"\n", i)
            k = n if k < 0 else k
            seq += data[i:k]
            if len(seq) > 1 and seq[-1] == ord("\r"):
                seq.pop()
            i = k + 1
        if i < n and data[i] in b">@":
            pending = True
            i += 1
        recs.append((name, bytes(seq)))
        if i >= n:
            return recs


def fasta_blocks(data: bytes, block_size: int = 500_000_000):
    """Blocks of src/main.cpp:336-455/486-528 -> (text, chroms [(name, start, len)], blocks [(start, len)])."""
    text = bytearray()
    chroms, blocks = [], []
    bstart, blen = 0, 0
    for name, seq in fasta_records(data):
        chroms.append((name, len(text), len(seq)))
        text += seq
        blen += len(seq)
        if blen > block_size:
            blocks.append((bstart, blen))
            bstart, blen = len(text), 0
        else:
            text += b"&"
            blen += 1
    if blen > 0:
        blocks.append((bstart, blen - 1))
    return bytes(text), chroms, blocks
