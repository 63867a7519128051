"""segalign_b200 — B200-native seed-filter path of SegAlign behind its C ABI.

The compute path is the CUDA library ``libsegalign_b200.so`` (kernels for
sm_100a + host C++).  This module is a thin ctypes binding that mirrors the
reference's ``seed_filter_interface`` call sequence (src/main.cpp:290-291,
606-674; src/seeder.cpp:78,113):

    sf = SeedFilter()
    sf.initialize_interface(-1)                       # InitializeInterface
    sf.generate_shape_pos("12of19")                  # GenerateShapePos
    sf.initialize_processor(transition, 250000, 19, sub_mat, 910, 3000, False)
    sf.send_ref_write_request(target_text)           # SendRefWriteRequest
    sf.generate_seed_pos_table(target_text, 1, 19, 12)   # GenerateSeedPosTable
    sf.send_query_write_request(query_text, 0)       # SendQueryWriteRequest
    hsps = sf.seed_and_filter(seeds, rev, 0)         # SeedAndFilter
    ...

There is no CPU fallback: importing works without a GPU, but every call that
computes needs the CUDA library and a device, and fails loudly otherwise.
"""
from __future__ import annotations

import ctypes as C
import os
import threading
import weakref

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsegalign_b200.so")

SEGMENT_DTYPE = np.dtype([("ref_start", "<u4"), ("query_start", "<u4"), ("len", "<u4"), ("score", "<i4")])

SA_OK = 0
ERRORS = {
    -1: "SA_ERR_ARG", -2: "SA_ERR_STATE", -3: "SA_ERR_CUDA", -4: "SA_ERR_NOMEM", -5: "SA_ERR_MAX_SEEDS",
    -6: "SA_ERR_BAD_SEED", -7: "SA_ERR_MAX_HITS", -8: "SA_ERR_CAPACITY", -9: "SA_ERR_NO_DEVICE",
    -10: "SA_ERR_TOO_MANY_GPUS",
}

# Every entry point of include/segalign_b200.h and include/segalign_b200_host.h.
EXPORTS = [
    "sa_initialize_interface", "sa_send_ref_write_request", "sa_clear_ref", "sa_generate_shape_pos",
    "sa_generate_seed_pos_table", "sa_send_seed_pos_table", "sa_get_seed_pos_table", "sa_initialize_processor",
    "sa_send_query_write_request", "sa_seed_and_filter", "sa_clear_query", "sa_shutdown_processor",
    "sa_rm_send_query_write_request", "sa_rm_seed_and_filter", "sa_rm_clear_query", "sa_free_segments",
    "sa_set_max_hits", "sa_set_rm_exclude_diagonal", "sa_last_call_stats", "sa_last_error", "sa_set_tuning",
    "sa_host_set_shape", "sa_host_chunk_seeds", "sa_host_revcomp", "sa_build_sub_mat", "sa_seeder_run",
    "sa_seed_and_filter_batch", "sa_set_timing", "sa_kernel_launches", "sa_seed_and_filter_noalloc",
    "sa_set_tuning_param", "sa_get_tuning_param",
    "sa_serve_start", "sa_serve_submit", "sa_serve_wait", "sa_serve_stop", "sa_autotune", "sa_get_timing",
    "sa_rm_seeder_run", "sa_free_rm_runs", "sa_format_segments", "sa_format_rm_intervals", "sa_free_text",
    "sa_fasta_load", "sa_seq_set_free", "sa_align_fasta", "sa_refresh_query_keys", "sa_format_segments_gpu",
]


class SegAlignError(RuntimeError):
    def __init__(self, code: int, fn: str, msg: str):
        super().__init__(f"{fn} -> {ERRORS.get(code, code)}: {msg}")
        self.code = code


class CallStats(C.Structure):
    _fields_ = [("num_seeds", C.c_uint64), ("num_hits", C.c_uint64), ("hits_extended", C.c_uint64),
                ("seeds_with_hits", C.c_uint64), ("survivors", C.c_uint64), ("num_hsps", C.c_uint64),
                ("long_hits", C.c_uint64), ("tiles", C.c_uint64), ("num_iter", C.c_uint32), ("batch_calls", C.c_uint32),
                ("ms_total", C.c_double), ("ms_lookup", C.c_double), ("ms_extend_lane", C.c_double),
                ("ms_extend_warp", C.c_double), ("ms_dedup", C.c_double), ("ms_copy", C.c_double)]


class SeederCfg(C.Structure):
    _fields_ = [("interval_size", C.c_uint32), ("interval_overlap", C.c_uint32), ("chunk_size", C.c_uint32),
                ("strand", C.c_int32), ("num_threads", C.c_int32), ("buffer", C.c_uint32),
                ("max_chunks", C.c_uint32), ("pad", C.c_uint32)]


class Unit(C.Structure):
    """sa_unit: seed positions [start, end) of query buffer `buffer` on strand `rev`."""
    _fields_ = [("buffer", C.c_uint32), ("rev", C.c_int32), ("start", C.c_uint32), ("end", C.c_uint32)]


class ServeCfg(C.Structure):
    """sa_serve_cfg: unit cutting, strands, seed slots per device pass, HBM left unused by admission."""
    _fields_ = [("interval_size", C.c_uint32), ("interval_overlap", C.c_uint32), ("chunk_size", C.c_uint32),
                ("strands", C.c_int32), ("pass_slots", C.c_uint64), ("hbm_reserve", C.c_uint64)]


class ServeStats(C.Structure):
    """sa_serve_request_stats: times in seconds since sa_serve_start."""
    _fields_ = [("submit_s", C.c_double), ("admit_s", C.c_double), ("done_s", C.c_double),
                ("num_units", C.c_uint64), ("num_passes", C.c_uint64), ("num_hits", C.c_uint64),
                ("num_hsps", C.c_uint64), ("device_bytes", C.c_uint64)]


SA_PENDING = 1


class AutotuneCfg(C.Structure):
    _fields_ = [("cache_path", C.c_char_p), ("repeats", C.c_int32), ("quick", C.c_int32), ("refresh", C.c_int32),
                ("pad", C.c_int32)]


class AutotuneResult(C.Structure):
    _fields_ = [("ext_ctas_per_sm", C.c_int32), ("step_bases", C.c_int32), ("tile_hits", C.c_int32),
                ("lane_cap", C.c_int32), ("range_ctas", C.c_int32), ("substeps", C.c_int32), ("switch_now", C.c_int32),
                ("candidates", C.c_int32),
                ("rejected", C.c_int32), ("from_cache", C.c_int32), ("ms_start", C.c_double),
                ("ms_best", C.c_double)]


class RmSeederCfg(C.Structure):
    _fields_ = [("lastz_interval_size", C.c_uint32), ("seq_block_size", C.c_uint32),
                ("prop_neigh_interval", C.c_float), ("M", C.c_uint32), ("chunk_size", C.c_uint32),
                ("strand", C.c_int32), ("num_threads", C.c_int32), ("max_intervals", C.c_uint32),
                ("step", C.c_uint32), ("pad", C.c_uint32)]


class RmSeederStats(C.Structure):
    _fields_ = [("num_seeds", C.c_uint64), ("num_hits", C.c_uint64), ("num_hsps", C.c_uint64),
                ("num_calls", C.c_uint64), ("num_intervals", C.c_uint64), ("num_blocks", C.c_uint64),
                ("seconds", C.c_double)]


class ChromTable(C.Structure):
    _fields_ = [("names", C.POINTER(C.c_char_p)), ("starts", C.POINTER(C.c_uint64)), ("lens", C.POINTER(C.c_uint32)),
                ("count", C.c_uint32), ("pad", C.c_uint32)]


def _chrom_table(chroms):
    """[(name, global start, length), ...] -> (ChromTable, kept buffers)."""
    names = (C.c_char_p * len(chroms))(*[c[0].encode() for c in chroms])
    starts = (C.c_uint64 * len(chroms))(*[int(c[1]) for c in chroms])
    lens = (C.c_uint32 * len(chroms))(*[int(c[2]) for c in chroms])
    return ChromTable(names, starts, lens, len(chroms), 0), (names, starts, lens)


RM_RUN_DTYPE = np.dtype([("block", "<u4"), ("interval", "<u4"), ("query_start", "<u4"), ("len", "<u4")])


class SeederStats(C.Structure):
    _fields_ = [("num_seeds", C.c_uint64), ("num_hits", C.c_uint64), ("num_hsps", C.c_uint64),
                ("num_calls", C.c_uint64), ("seconds", C.c_double), ("seed_seconds", C.c_double),
                ("call_seconds", C.c_double), ("copy_seconds", C.c_double)]


class SeqSet(C.Structure):
    _fields_ = [("text", C.c_void_p), ("text_len", C.c_uint64), ("num_chroms", C.c_uint32),
                ("num_blocks", C.c_uint32), ("names", C.POINTER(C.c_char_p)), ("chrom_start", C.POINTER(C.c_uint64)),
                ("chrom_len", C.POINTER(C.c_uint32)), ("block_start", C.POINTER(C.c_uint64)),
                ("block_len", C.POINTER(C.c_uint32)), ("impl", C.c_void_p)]


class AlignCfg(C.Structure):
    _fields_ = [("target_path", C.c_char_p), ("query_path", C.c_char_p), ("segments_path", C.c_char_p),
                ("hsp_path", C.c_char_p), ("seq_block_size", C.c_uint32), ("interval_size", C.c_uint32),
                ("interval_overlap", C.c_uint32), ("chunk_size", C.c_uint32), ("strand", C.c_int32),
                ("num_threads", C.c_int32), ("step", C.c_uint32), ("pad", C.c_uint32)]


class AlignStats(C.Structure):
    _fields_ = [("ref_blocks", C.c_uint64), ("query_blocks", C.c_uint64), ("intervals", C.c_uint64),
                ("num_seeds", C.c_uint64), ("num_hits", C.c_uint64), ("num_hsps", C.c_uint64),
                ("seconds", C.c_double), ("read_seconds", C.c_double), ("table_seconds", C.c_double),
                ("query_write_seconds", C.c_double), ("overlap_seconds", C.c_double), ("calls_seconds", C.c_double),
                ("output_seconds", C.c_double)]


_lib = None
_lib_lock = threading.Lock()
_P = C.POINTER


def load_library(path: str = LIB_PATH) -> C.CDLL:
    """Loads the CUDA library; raises if it has not been built."""
    global _lib
    with _lib_lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: build it with `python -m segalign_b200._build` "
                               "(there is no CPU fallback)")
        lib = C.CDLL(path)
        u64p, u32p, i32p = _P(C.c_uint64), _P(C.c_uint32), _P(C.c_int32)
        segpp = _P(_P(C.c_uint8))
        sig = {
            "sa_initialize_interface": (C.c_int, [C.c_int]),
            "sa_send_ref_write_request": (C.c_int, [C.c_char_p, C.c_size_t, C.c_uint32]),
            "sa_clear_ref": (C.c_int, []),
            "sa_generate_shape_pos": (C.c_int, [C.c_char_p]),
            "sa_generate_seed_pos_table": (C.c_int, [C.c_char_p, C.c_size_t, C.c_uint32, C.c_uint32, C.c_int, C.c_int]),
            "sa_send_seed_pos_table": (C.c_int, [u32p, C.c_uint32, u32p, C.c_uint32]),
            "sa_get_seed_pos_table": (C.c_int, [u32p, C.c_uint64, u32p, C.c_uint64, u64p, u64p]),
            "sa_initialize_processor": (C.c_int, [C.c_int, C.c_uint32, C.c_uint32, i32p, C.c_int, C.c_int, C.c_int]),
            "sa_send_query_write_request": (C.c_int, [C.c_char_p, C.c_size_t, C.c_uint32, C.c_uint32]),
            "sa_seed_and_filter": (C.c_int, [u64p, C.c_uint32, C.c_int, C.c_uint32, segpp, u64p]),
            "sa_clear_query": (C.c_int, [C.c_uint32]),
            "sa_shutdown_processor": (C.c_int, []),
            "sa_rm_send_query_write_request": (C.c_int, []),
            "sa_rm_seed_and_filter": (C.c_int, [u64p, C.c_uint32, C.c_int, C.c_uint32, C.c_uint32, segpp, u64p]),
            "sa_rm_clear_query": (C.c_int, []),
            "sa_free_segments": (None, [_P(C.c_uint8)]),
            "sa_set_max_hits": (C.c_int, [C.c_uint64]),
            "sa_set_rm_exclude_diagonal": (C.c_int, [C.c_int]),
            "sa_last_call_stats": (C.c_int, [_P(CallStats)]),
            "sa_last_error": (C.c_char_p, []),
            "sa_set_tuning": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int]),
            "sa_host_set_shape": (C.c_int, [C.c_char_p, C.c_int]),
            "sa_host_chunk_seeds": (C.c_uint64, [C.c_char_p, C.c_uint32, C.c_uint32, u64p, C.c_uint64]),
            "sa_host_revcomp": (C.c_uint64, [C.c_char_p, C.c_char_p, C.c_uint64]),
            "sa_build_sub_mat": (C.c_int, [C.c_int, C.c_char_p, i32p]),
            "sa_seeder_run": (C.c_int, [_P(SeederCfg), C.c_char_p, C.c_uint32, segpp, u64p, segpp, u64p,
                                        _P(SeederStats)]),
            "sa_seed_and_filter_batch": (C.c_int, [_P(Unit), C.c_uint32, segpp, u64p, u64p]),
            "sa_set_timing": (C.c_int, [C.c_int]),
            "sa_set_tuning_param": (C.c_int, [C.c_char_p, C.c_int]),
            "sa_get_tuning_param": (C.c_int, [C.c_char_p]),
            "sa_seed_and_filter_noalloc": (C.c_int, [u64p, C.c_uint32, C.c_int, C.c_uint32, _P(C.c_uint8),
                                                     C.c_uint64, u64p]),
            "sa_kernel_launches": (C.c_uint64, []),
            "sa_fasta_load": (C.c_int, [C.c_char_p, C.c_uint32, _P(SeqSet)]),
            "sa_refresh_query_keys": (C.c_int, [C.c_uint32]),
            "sa_seq_set_free": (None, [_P(SeqSet)]),
            "sa_align_fasta": (C.c_int, [_P(AlignCfg), _P(AlignStats)]),
            "sa_serve_start": (C.c_int, [_P(ServeCfg)]),
            "sa_serve_submit": (C.c_int, [C.c_char_p, C.c_uint32, u64p]),
            "sa_serve_wait": (C.c_int, [C.c_uint64, C.c_int, segpp, u64p, segpp, u64p, _P(ServeStats)]),
            "sa_serve_stop": (C.c_int, []),
            "sa_autotune": (C.c_int, [_P(Unit), C.c_uint32, _P(AutotuneCfg), _P(AutotuneResult)]),
            "sa_get_timing": (C.c_int, []),
            "sa_rm_seeder_run": (C.c_int, [_P(RmSeederCfg), C.c_char_p, C.c_uint64, _P(_P(C.c_uint8)), u64p,
                                           _P(RmSeederStats)]),
            "sa_free_rm_runs": (None, [_P(C.c_uint8)]),
            "sa_format_segments": (C.c_int, [_P(ChromTable), C.c_uint64, _P(ChromTable), C.c_uint64, C.c_uint32,
                                             _P(C.c_uint8), C.c_uint64, _P(C.c_uint8), C.c_uint64,
                                             _P(C.c_void_p), u64p, _P(C.c_void_p), u64p]),
            "sa_format_segments_gpu": (C.c_int, [_P(ChromTable), C.c_uint64, _P(ChromTable), C.c_uint64, C.c_uint32,
                                             _P(C.c_uint8), C.c_uint64, _P(C.c_uint8), C.c_uint64,
                                             _P(C.c_void_p), u64p, _P(C.c_void_p), u64p]),
            "sa_format_rm_intervals": (C.c_int, [_P(ChromTable), C.c_uint64, _P(C.c_uint8), C.c_uint64, C.c_int,
                                                 _P(C.c_void_p), u64p]),
            "sa_free_text": (None, [C.c_void_p]),
        }
        for name, (res, args) in sig.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
        return lib


def _u64p(a: np.ndarray):
    return a.ctypes.data_as(_P(C.c_uint64))


def _u32p(a: np.ndarray):
    return a.ctypes.data_as(_P(C.c_uint32))


def _bytes(text) -> bytes:
    if isinstance(text, np.ndarray):
        return text.tobytes()
    if isinstance(text, str):
        return text.encode("ascii")
    return bytes(text)


def build_sub_mat(xdrop: int = 910, ambiguous: str = "") -> np.ndarray:
    """Scoring table of src/main.cpp:180-261 (C++ host code)."""
    lib = load_library()
    m = np.zeros(64, dtype=np.int32)
    r = lib.sa_build_sub_mat(xdrop, ambiguous.encode(), m.ctypes.data_as(_P(C.c_int32)))
    if r != SA_OK:
        raise SegAlignError(r, "sa_build_sub_mat", "bad ambiguous string")
    return m


def host_seeds(text: bytes, j0: int, j1: int, shape: str = "12of19", transition: bool = False) -> np.ndarray:
    """Seed words of query positions [j0, j1) (src/seeder.cpp:57-74), computed by the C++ host seeder."""
    lib = load_library()
    lib.sa_host_set_shape(shape.encode(), int(transition))
    n = lib.sa_host_chunk_seeds(text, j0, j1, None, 0)
    out = np.empty(max(n, 1), dtype=np.uint64)
    lib.sa_host_chunk_seeds(text, j0, j1, _u64p(out), n)
    return out[:n]


def host_revcomp(text: bytes) -> bytes:
    lib = load_library()
    dst = C.create_string_buffer(len(text))
    n = lib.sa_host_revcomp(dst, text, len(text))
    return dst.raw[:n]


def _take_segments(lib, ptr, n) -> np.ndarray:
    """The library's malloc'd HSP array as a numpy array, without a copy: the
    buffer is freed (sa_free_segments) when the array is garbage-collected."""
    if n == 0:
        lib.sa_free_segments(ptr)
        return np.zeros(0, dtype=SEGMENT_DTYPE)
    raw = np.ctypeslib.as_array(C.cast(ptr, _P(C.c_uint8)), shape=(16 * n,))
    weakref.finalize(raw, lib.sa_free_segments, C.cast(ptr, _P(C.c_uint8)))
    return raw.view(SEGMENT_DTYPE)


class SeedFilter:
    """Mirror of the reference seed_filter_interface over the C ABI."""

    def __init__(self):
        self.lib = load_library()

    def _chk(self, r: int, fn: str) -> int:
        if r < 0:
            raise SegAlignError(r, fn, (self.lib.sa_last_error() or b"").decode())
        return r

    # ---- common/seed_filter_interface.cu ----
    def initialize_interface(self, num_gpu: int = -1) -> int:
        return self._chk(self.lib.sa_initialize_interface(num_gpu), "InitializeInterface")

    def send_ref_write_request(self, seq, start_addr: int = 0, length: int | None = None) -> None:
        self._ref = _bytes(seq)
        n = len(self._ref) - start_addr if length is None else length
        self._chk(self.lib.sa_send_ref_write_request(self._ref, start_addr, n), "SendRefWriteRequest")
        self._ref_args = (start_addr, n)

    def clear_ref(self) -> None:
        self._chk(self.lib.sa_clear_ref(), "ClearRef")

    # ---- seeds and table ----
    def generate_shape_pos(self, shape: str = "12of19") -> int:
        return self._chk(self.lib.sa_generate_shape_pos(shape.encode()), "GenerateShapePos")

    def generate_seed_pos_table(self, ref=None, step: int = 1, shape_size: int = 19, kmer_size: int = 12,
                                start_addr: int | None = None, length: int | None = None) -> None:
        if ref is None:
            ref = self._ref
            s, n = self._ref_args
        else:
            ref = _bytes(ref)
            if ref == getattr(self, "_ref", None):
                ref = self._ref  # same host buffer -> build from the resident target
            s = 0 if start_addr is None else start_addr
            n = len(ref) - s if length is None else length
        self._chk(self.lib.sa_generate_seed_pos_table(ref, s, n, step, shape_size, kmer_size), "GenerateSeedPosTable")

    def send_seed_pos_table(self, index_table: np.ndarray, pos_table: np.ndarray) -> None:
        it = np.ascontiguousarray(index_table, dtype=np.uint32)
        pt = np.ascontiguousarray(pos_table, dtype=np.uint32)
        self._chk(self.lib.sa_send_seed_pos_table(_u32p(it), len(it), _u32p(pt), len(pt)), "SendSeedPosTable")

    def get_seed_pos_table(self):
        nb, ni = C.c_uint64(), C.c_uint64()
        self._chk(self.lib.sa_get_seed_pos_table(None, 0, None, 0, C.byref(nb), C.byref(ni)), "GetSeedPosTable")
        it = np.empty(nb.value, dtype=np.uint32)
        pt = np.empty(max(ni.value, 1), dtype=np.uint32)
        self._chk(self.lib.sa_get_seed_pos_table(_u32p(it), nb.value, _u32p(pt), ni.value, None, None),
                  "GetSeedPosTable")
        return it, pt[: ni.value]

    # ---- src/seed_filter.cu ----
    def initialize_processor(self, transition: bool, wga_chunk: int, seed_size: int, sub_mat, xdrop: int,
                             hspthresh: int, noentropy: bool) -> None:
        m = np.ascontiguousarray(sub_mat, dtype=np.int32)
        self._chk(self.lib.sa_initialize_processor(int(transition), wga_chunk, seed_size,
                                                   m.ctypes.data_as(_P(C.c_int32)), xdrop, hspthresh,
                                                   int(noentropy)), "InitializeProcessor")

    def send_query_write_request(self, query, buffer: int = 0, start_addr: int = 0, length: int | None = None):
        q = _bytes(query)
        n = len(q) - start_addr if length is None else length
        self._chk(self.lib.sa_send_query_write_request(q, start_addr, n, buffer), "SendQueryWriteRequest")

    def seed_and_filter(self, seeds: np.ndarray, rev: bool, buffer: int = 0) -> np.ndarray:
        s = np.ascontiguousarray(seeds, dtype=np.uint64)
        ptr, n = _P(C.c_uint8)(), C.c_uint64()
        self._chk(self.lib.sa_seed_and_filter(_u64p(s), len(s), int(rev), buffer, C.byref(ptr), C.byref(n)),
                  "SeedAndFilter")
        return _take_segments(self.lib, ptr, n.value)

    def seed_and_filter_noalloc(self, seeds: np.ndarray, rev: bool, buffer: int = 0,
                                out: np.ndarray | None = None) -> np.ndarray:
        """SeedAndFilter without allocation: the result goes into `out` (SEGMENT_DTYPE records)."""
        s = np.ascontiguousarray(seeds, dtype=np.uint64)
        if out is None:
            out = np.zeros(1 << 16, dtype=SEGMENT_DTYPE)
        n = C.c_uint64()
        self._chk(self.lib.sa_seed_and_filter_noalloc(_u64p(s), len(s), int(rev), buffer,
                                                      out.ctypes.data_as(_P(C.c_uint8)), len(out), C.byref(n)),
                  "SeedAndFilterNoAlloc")
        return out[: n.value].copy()

    def clear_query(self, buffer: int = 0) -> None:
        self._chk(self.lib.sa_clear_query(buffer), "ClearQuery")

    def shutdown_processor(self) -> None:
        self._chk(self.lib.sa_shutdown_processor(), "ShutdownProcessor")

    def refresh_query_keys(self, buffer: int = 0) -> None:
        """Recomputes the per-position keys of a resident query buffer on the GPU."""
        self._chk(self.lib.sa_refresh_query_keys(buffer), "refresh_query_keys")

    def seed_and_filter_batch(self, units, keep_on_device: bool = False):
        """Batched form: units = [(buffer, rev, start, end), ...].

        Returns one header+HSP array per unit (as seed_and_filter would for the
        host seeds of that window), or None with keep_on_device=True.
        """
        arr = (Unit * max(len(units), 1))(*[Unit(b, int(r), s, e) for (b, r, s, e) in units])
        if keep_on_device:
            self._chk(self.lib.sa_seed_and_filter_batch(arr, len(units), None, None, None), "SeedAndFilterBatch")
            return None
        ptr, n = _P(C.c_uint8)(), C.c_uint64()
        offs = np.zeros(len(units) + 1, dtype=np.uint64)
        self._chk(self.lib.sa_seed_and_filter_batch(arr, len(units), C.byref(ptr), C.byref(n), _u64p(offs)),
                  "SeedAndFilterBatch")
        allsegs = _take_segments(self.lib, ptr, n.value)
        return [allsegs[int(offs[i]):int(offs[i + 1])] for i in range(len(units))]

    def autotune(self, units, cache_path: str | None = None, repeats: int = 0, quick: bool = False,
                 refresh: bool = False) -> dict:
        """Picks the fastest tuning for a batch of units (sa_autotune) and applies it."""
        arr = (Unit * max(len(units), 1))(*[Unit(b, int(r), s, e) for (b, r, s, e) in units])
        cfg = AutotuneCfg(cache_path.encode() if cache_path else None, repeats, int(quick), int(refresh), 0)
        res = AutotuneResult()
        self._chk(self.lib.sa_autotune(arr, len(units), C.byref(cfg), C.byref(res)), "autotune")
        return {k: getattr(res, k) for k, _ in AutotuneResult._fields_}

    def rm_seeder_run(self, seq, lastz_interval_size: int = 0, seq_block_size: int = 0, prop: float = 0.0,
                      M: int = 0, chunk_size: int = 0, strand: int = 3, num_threads: int = 4,
                      max_intervals: int = 0, step: int = 1, shape: str = "12of19", transition: bool = False):
        """Repeat-masker self-alignment over a whole sequence (sa_rm_seeder_run):
        (runs as RM_RUN_DTYPE records, stats)."""
        q = _bytes(seq)
        self.lib.sa_host_set_shape(shape.encode(), int(transition))
        cfg = RmSeederCfg(lastz_interval_size, seq_block_size, prop, M, chunk_size, strand, num_threads,
                          max_intervals, step, 0)
        ptr, n, st = _P(C.c_uint8)(), C.c_uint64(), RmSeederStats()
        self._chk(self.lib.sa_rm_seeder_run(C.byref(cfg), q, len(q), C.byref(ptr), C.byref(n), C.byref(st)),
                  "rm_seeder_run")
        try:
            runs = np.frombuffer(bytes(C.cast(ptr, _P(C.c_uint8 * (16 * n.value))).contents), dtype=RM_RUN_DTYPE).copy() \
                if n.value else np.zeros(0, dtype=RM_RUN_DTYPE)
        finally:
            self.lib.sa_free_rm_runs(ptr)
        return runs, {k: getattr(st, k) for k, _ in RmSeederStats._fields_}

    # ---- repeat_masker_src/seed_filter.cu ----
    def rm_send_query_write_request(self) -> None:
        self._chk(self.lib.sa_rm_send_query_write_request(), "SendQueryWriteRequest(rm)")

    def rm_seed_and_filter(self, seeds: np.ndarray, rev: bool, ref_start: int, ref_end: int) -> np.ndarray:
        s = np.ascontiguousarray(seeds, dtype=np.uint64)
        ptr, n = _P(C.c_uint8)(), C.c_uint64()
        self._chk(self.lib.sa_rm_seed_and_filter(_u64p(s), len(s), int(rev), ref_start, ref_end, C.byref(ptr),
                                                 C.byref(n)), "SeedAndFilter(rm)")
        return _take_segments(self.lib, ptr, n.value)

    def rm_clear_query(self) -> None:
        self._chk(self.lib.sa_rm_clear_query(), "ClearQuery(rm)")

    # ---- configuration / diagnostics ----
    def set_max_hits(self, n: int) -> None:
        self._chk(self.lib.sa_set_max_hits(n), "set_max_hits")

    def set_rm_exclude_diagonal(self, on: bool) -> None:
        self._chk(self.lib.sa_set_rm_exclude_diagonal(int(on)), "set_rm_exclude_diagonal")

    def set_tuning(self, lane_cap=-1, ext_block=-1, ext_ctas_per_sm=-1, tile_hits=-1, **named) -> None:
        for k, v in named.items():  # step_bases, range_ctas
            self._chk(self.lib.sa_set_tuning_param(k.encode(), int(v)), f"set_tuning({k})")
        self._chk(self.lib.sa_set_tuning(lane_cap, ext_block, ext_ctas_per_sm, tile_hits), "set_tuning")

    def get_tuning(self) -> dict:
        names = ("lane_cap", "ext_ctas_per_sm", "tile_hits", "step_bases", "range_ctas", "substeps", "call_range_ctas",
                 "call_lane_ctas", "switch_now", "rm_lane_ctas", "rm_substeps", "rm_switch_now")
        return {n: int(self.lib.sa_get_tuning_param(n.encode())) for n in names}

    def set_timing(self, on: bool) -> None:
        self.lib.sa_set_timing(int(on))

    def kernel_launches(self) -> int:
        return int(self.lib.sa_kernel_launches())

    def last_call_stats(self) -> dict:
        st = CallStats()
        self.lib.sa_last_call_stats(C.byref(st))
        return {k: getattr(st, k) for k, _ in CallStats._fields_ if k != "pad"}

    # ---- serving form ----
    def serve_start(self, interval_size: int = 10_000_000, interval_overlap: int = 0, chunk_size: int = 0,
                    strands: int = 3, pass_slots: int = 0, hbm_reserve: int = 0) -> None:
        """Starts the request loop over the resident target (sa_serve_start)."""
        cfg = ServeCfg(interval_size, interval_overlap, chunk_size, strands, pass_slots, hbm_reserve)
        self._chk(self.lib.sa_serve_start(C.byref(cfg)), "serve_start")

    def serve_submit(self, query) -> int:
        """Queues one query sequence; returns its request id."""
        q = _bytes(query)
        rid = C.c_uint64()
        self._chk(self.lib.sa_serve_submit(q, len(q), C.byref(rid)), "serve_submit")
        return rid.value

    def serve_wait(self, request_id: int, timeout_ms: int = -1):
        """(plus HSPs, minus HSPs, stats) of a request, or None if it is not
        finished within timeout_ms; raises SegAlignError if it failed."""
        fw, fl, rc, rl = _P(C.c_uint8)(), C.c_uint64(), _P(C.c_uint8)(), C.c_uint64()
        st = ServeStats()
        r = self.lib.sa_serve_wait(request_id, timeout_ms, C.byref(fw), C.byref(fl), C.byref(rc), C.byref(rl),
                                   C.byref(st))
        if r == SA_PENDING:
            return None
        self._chk(r, "serve_wait")
        f = _take_segments(self.lib, fw, fl.value)
        g = _take_segments(self.lib, rc, rl.value)
        return f, g, {k: getattr(st, k) for k, _ in ServeStats._fields_}

    def serve_stop(self) -> None:
        self._chk(self.lib.sa_serve_stop(), "serve_stop")

    def align_fasta(self, target_path: str, query_path: str, segments_path: str | None = None,
                    hsp_path: str | None = None, seq_block_size: int = 0, interval_size: int = 0,
                    interval_overlap: int = 0, chunk_size: int = 0, strand: int = 3, num_threads: int = 0,
                    step: int = 1, shape: str = "12of19", transition: bool = False) -> dict:
        """Whole-file driver (sa_align_fasta): target blocks, double-buffered query blocks, segments out."""
        self.lib.sa_host_set_shape(shape.encode(), int(transition))
        enc = lambda x: x.encode() if x else None  # noqa: E731
        cfg = AlignCfg(enc(target_path), enc(query_path), enc(segments_path), enc(hsp_path), seq_block_size,
                       interval_size, interval_overlap, chunk_size, strand, num_threads, step, 0)
        st = AlignStats()
        self._chk(self.lib.sa_align_fasta(C.byref(cfg), C.byref(st)), "align_fasta")
        return {k: getattr(st, k) for k, _ in AlignStats._fields_}

    def seeder_run(self, query, buffer: int = 0, strand: int = 3, num_threads: int = 4,
                   interval_size: int = 10_000_000, chunk_size: int = 250_000, interval_overlap: int = 0,
                   max_chunks: int = 0, shape: str = "12of19", transition: bool = False):
        """Seeder pipeline over one query block (src/seeder.cpp:12-127) in C++ host threads."""
        q = _bytes(query)
        self.lib.sa_host_set_shape(shape.encode(), int(transition))
        cfg = SeederCfg(interval_size, interval_overlap, chunk_size, strand, num_threads, buffer, max_chunks, 0)
        fw, fl, rc, rl = _P(C.c_uint8)(), C.c_uint64(), _P(C.c_uint8)(), C.c_uint64()
        st = SeederStats()
        self._chk(self.lib.sa_seeder_run(C.byref(cfg), q, len(q), C.byref(fw), C.byref(fl), C.byref(rc),
                                         C.byref(rl), C.byref(st)), "seeder_run")
        f = _take_segments(self.lib, fw, fl.value)
        r = _take_segments(self.lib, rc, rl.value)
        return f, r, {k: getattr(st, k) for k, _ in SeederStats._fields_}


def fasta_load(path: str, seq_block_size: int = 0) -> dict:
    """A FASTA file joined into '&'-separated blocks (sa_fasta_load):
    {"text": bytes, "chroms": [(name, start, len)], "blocks": [(start, len)]}."""
    lib = load_library()
    ss = SeqSet()
    st = lib.sa_fasta_load(path.encode(), seq_block_size, C.byref(ss))
    if st != 0:
        raise SegAlignError(st, "fasta_load", (lib.sa_last_error() or b"").decode())
    try:
        text = C.string_at(ss.text, ss.text_len) if ss.text_len else b""
        chroms = [(ss.names[i].decode(), ss.chrom_start[i], ss.chrom_len[i]) for i in range(ss.num_chroms)]
        blocks = [(ss.block_start[i], ss.block_len[i]) for i in range(ss.num_blocks)]
    finally:
        lib.sa_seq_set_free(C.byref(ss))
    return {"text": text, "chroms": chroms, "blocks": blocks}


def _take_text(lib, ptr: C.c_void_p, n: int) -> str:
    try:
        return C.string_at(ptr, n).decode() if n else ""
    finally:
        lib.sa_free_text(ptr)


def format_segments(ref_chroms, ref_block_start: int, query_chroms, query_block_start: int, query_block_len: int,
                    fw: np.ndarray, rc: np.ndarray, gpu: bool = False):
    """lastz --segments lines of one interval's HSP lists (sa_format_segments,
    or sa_format_segments_gpu with gpu=True; the same text): (plus-strand
    text, minus-strand text).  Chromosome tables are [(name, global start,
    length), ...]."""
    lib = load_library()
    rt, keep1 = _chrom_table(ref_chroms)
    qt, keep2 = _chrom_table(query_chroms)
    f = np.ascontiguousarray(fw, dtype=SEGMENT_DTYPE)
    r = np.ascontiguousarray(rc, dtype=SEGMENT_DTYPE)
    pt, pl, mt, ml = C.c_void_p(), C.c_uint64(), C.c_void_p(), C.c_uint64()
    fn = lib.sa_format_segments_gpu if gpu else lib.sa_format_segments
    st = fn(C.byref(rt), ref_block_start, C.byref(qt), query_block_start, query_block_len,
            f.ctypes.data_as(_P(C.c_uint8)), len(f), r.ctypes.data_as(_P(C.c_uint8)), len(r),
            C.byref(pt), C.byref(pl), C.byref(mt), C.byref(ml))
    if st != 0:
        raise SegAlignError(st, "format_segments", "")
    return _take_text(lib, pt, pl.value), _take_text(lib, mt, ml.value)


def format_rm_intervals(chroms, block_start: int, runs: np.ndarray, markend: bool = False) -> str:
    """Repeat-masker interval lines of one interval's runs (sa_format_rm_intervals)."""
    lib = load_library()
    ct, keep = _chrom_table(chroms)
    r = np.ascontiguousarray(runs, dtype=RM_RUN_DTYPE)
    t, n = C.c_void_p(), C.c_uint64()
    st = lib.sa_format_rm_intervals(C.byref(ct), block_start, r.ctypes.data_as(_P(C.c_uint8)), len(r), int(markend),
                                    C.byref(t), C.byref(n))
    if st != 0:
        raise SegAlignError(st, "format_rm_intervals", "")
    return _take_text(lib, t, n.value)
