#!/usr/bin/env python
"""Benchmark of the B200 seed-filter path: ungapped extensions/s (and HSPs/s).

Workload (named by its sizes): genome scale, a synthetic 100 Mbp target in 6
chromosomes against a 108 Mbp query, GC 36%, ~60% of the query built from
target blocks of 1-50 kbp at 15-35% divergence (5% inverted), 12% repeats,
8% soft-masking.  12of19 seed, no transitions, HOXD70, xdrop 910, hspthresh
3000, entropy on, both strands; query intervals of 10 Mbp with 50 kbp
overlap cut into 250 kbp SeedAndFilter units.

One step = one pass of the hot path over the whole query (both strands):
  value  batched form, target table + query text resident in HBM: device
         seeding (per-position keys recomputed every step), lookup, X-drop,
         dedup, and the HSP lists copied to the host per unit; CUDA events
         on the current stream bracket each step (the calls return once the
         lists are on the host; device-only event time of the library's
         stream beside it);
  e2e    the reference-facing C ABI: the C++ seeder builds each unit's seed
         words on the host and calls sa_seed_and_filter(), which copies them to
         the GPU and copies the HSP list back (host wall time);
  e2e_batched  host query text -> GPU -> batched call -> HSP lists on the host.
Beside them: like-for-like batched/plain ratios, uneven windows, serving on
the resident table, an unranked timing of the reference's own kernels on a
sample of the same units, the CPU port on a bounded sample, the same workload
as FASTA files through sa_align_fasta to a segments file, and the 600 Mbp
legs (batched and plain with transitions, serving on that table, repeat-masker
self-alignment).  Ranks (torchrun) run one job: the target is replicated to
every GPU and the query is split, with no collective on the data path.  By
default (--scaling weak) the job's query is N blocks of the named size, drawn
from the one target, block r on rank r; --scaling strong splits the named
query into N slices.  value = all ranks' extensions / the slowest rank's time.

--impl reference times the reference semantics on the host cores (the CPU
port in oracle/), rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

INTERVAL, OVERLAP, CHUNK, SEED_SIZE = 10_000_000, 50_000, 250_000, 19
METRIC, UNIT = "ungapped extensions/s", "extensions/s"
FALLBACK_HBM_GBS = 6650.0


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--scale", type=float, default=1.0, help="workload size factor (1.0 = named sizes)")
    ap.add_argument("--scaling", choices=["weak", "strong"], default="weak",
                    help="N>1: weak = one query block of the named size per rank against the one target; "
                         "strong = the named query split across the ranks")
    ap.add_argument("--cpu-chunks", type=int, default=None,
                    help="units in the bounded CPU sample (default 64; 2 for --workload large)")
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving leg")
    ap.add_argument("--serve-requests", type=int, default=None,
                    help="requests per load in the genome serving leg (default 200)")
    ap.add_argument("--large-serve-requests", type=int, default=24,
                    help="requests per load in the serving leg on the 600 Mbp table")
    ap.add_argument("--no-large", action="store_true",
                    help="skip the 600 Mbp legs (batched and plain with transitions, serving, repeat masker)")
    ap.add_argument("--large-cpu-units", type=int, default=0,
                    help="units of the 600 Mbp leg also run through the CPU port (0 = none: its table build "
                         "takes minutes on the host)")
    ap.add_argument("--no-fasta", action="store_true",
                    help="skip the whole-file leg (the workload as FASTA through sa_align_fasta to a segments file)")
    ap.add_argument("--no-ref-gpu", action="store_true",
                    help="skip the unranked timing of the reference's own kernels (oracle/_ref)")
    ap.add_argument("--ref-gpu-units", type=int, default=16,
                    help="250 kbp units of the genome workload timed through the reference's own kernels")
    ap.add_argument("--workload", choices=["genome", "large"], default="genome",
                    help="genome: 100 Mbp x 108 Mbp (the headline); large: 600 Mbp x 600 Mbp with transitions, "
                         "a query sample of --query-sample bases against the whole target")
    ap.add_argument("--query-sample", type=int, default=12_000_000, help="query bases used by --workload large")
    ap.add_argument("--rm-intervals", type=int, default=8,
                    help="repeat-masker intervals run on the 600 Mbp target (0 = skip)")
    return ap.parse_args()


def seeder_calls(query_len: int):
    """SeedAndFilter calls in seeder order: per interval (src/main.cpp:373-386, plus a 50 kbp
    overlap), its plus-strand chunks then its minus-strand chunks (src/seeder.cpp:47-121)."""
    L = query_len - SEED_SIZE
    calls = []
    for s in range(0, L, INTERVAL):
        e = min(L, s + INTERVAL + OVERLAP)
        for i in range(s, e, CHUNK):
            calls.append((0, 0, i, min(i + CHUNK, e)))
        rs, re = L - e, L - s
        for i in range(rs, re, CHUNK):
            calls.append((0, 1, i, min(i + CHUNK, re)))
    return calls


def lane_traffic(hits: float, workload: str):
    """DRAM bytes (read + write) of one lane-kernel launch, scaled by hits from
    the ncu capture of this workload recorded in profiles/extend_lane_dram.json;
    (None, why) if there is none."""
    path = os.path.join(ROOT, "profiles", "extend_lane_dram.json")
    try:
        with open(path) as f:
            d = json.load(f)[workload]
        per_hit = float(d["dram_bytes"]) / float(d["hits"])
    except (OSError, KeyError, ValueError, ZeroDivisionError, TypeError):
        return None, f"no ncu capture recorded for the {workload} workload"
    return per_hit * hits, f"ncu dram bytes per hit of {d['workload']} x this launch's hits"


def lane_limit(workload: str):
    """The lane kernel's measured issue-bound limit (ncu full capture) recorded
    beside its DRAM traffic in profiles/extend_lane_dram.json, or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "extend_lane_dram.json")) as f:
            return json.load(f)[workload].get("issue")
    except (OSError, KeyError, ValueError):
        return None


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.idx), "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def gpu_index(local_rank: int) -> int:
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [x for x in vis.split(",") if x.strip()]
        if local_rank < len(ids) and ids[local_rank].strip().isdigit():
            return int(ids[local_rank])
    return local_rank


# ---------------------------------------------------------------------------
# CPU baseline (reference semantics on the host cores)
# ---------------------------------------------------------------------------
_TABLES = {}


def cpu_sample(w, max_chunks: int, threads: int, transition: bool = False):
    import oracle

    p = oracle.params(transition=transition)
    t = time.perf_counter()
    key = id(w)
    if key not in _TABLES:
        _TABLES[key] = oracle.build_table(w.target, p)
    idx, pos = _TABLES[key]
    table_s = time.perf_counter() - t
    t = time.perf_counter()
    fw, rc, st = oracle.pipeline(p, w.target, w.query, idx, pos, strand=3, nthreads=threads, interval_size=INTERVAL,
                                 chunk_size=CHUNK, interval_overlap=OVERLAP, max_chunks=max_chunks)
    dt = time.perf_counter() - t
    return dict(seconds=dt, hits=st["num_hits"], hsps=st["num_hsps"], table_s=table_s, fw=fw, rc=rc, stats=st)


def serve_requests(target: bytes, n: int, seed: int):
    """Request texts of the serving workload: lengths log-uniform in
    [10 kbp, 20 Mbp]; 30% of each request's bases are target blocks of
    1-50 kbp with 20% substitutions, the rest i.i.d. bases at GC 36%."""
    rng = np.random.default_rng(seed)
    tgt = np.frombuffer(target, dtype=np.uint8)
    acgt = np.frombuffer(b"ACGT", dtype=np.uint8)
    out = []
    for _ in range(n):
        L = int(np.exp(rng.uniform(np.log(1e4), np.log(2e7))))
        parts, have = [], 0
        while have < L:
            b = int(min(L - have, rng.integers(1_000, 50_001)))
            if rng.random() < 0.3:
                a = int(rng.integers(0, len(tgt) - b))
                blk = tgt[a:a + b].copy()
                m = rng.random(b) < 0.2
                blk[m] = acgt[rng.integers(0, 4, int(m.sum()))]
            else:
                blk = acgt[rng.choice(4, size=b, p=[0.32, 0.18, 0.18, 0.32])]
            parts.append(blk)
            have += b
        out.append(np.concatenate(parts).tobytes())
    return out


def distinct_rows(lists) -> np.ndarray:
    """Distinct HSP records (16-byte rows) of a list of HSP arrays, sorted."""
    a = np.concatenate([np.asarray(x).view(np.uint32).reshape(-1, 4) for x in lists]) if lists else \
        np.zeros((0, 4), dtype=np.uint32)
    k = a.view(np.uint64).reshape(-1, 2)
    order = np.lexsort((k[:, 1], k[:, 0]))
    k = k[order]
    keep = np.ones(len(k), dtype=bool)
    keep[1:] = (k[1:, 0] != k[:-1, 0]) | (k[1:, 1] != k[:-1, 1])
    return k[keep]


def run_uneven(sf, query_len: int, chunked_outs, chunked_units) -> dict:
    """Batched form over uneven query windows (log-uniform 50 kbp-10 Mbp, both
    strands, seeds 103/104): device time, and its distinct HSPs per strand
    against the 250 kbp-chunk run's (chunking only adds duplicates)."""
    from segalign_b200.synth import loguniform_chunks
    L = query_len - SEED_SIZE
    units = [(0, r, int(a), int(b)) for r in (0, 1) for a, b in loguniform_chunks(103 + r, L, 5e4, 1e7)]
    sf.set_timing(True)
    sf.seed_and_filter_batch(units, keep_on_device=True)  # warm
    ms = []
    for _ in range(3):
        sf.seed_and_filter_batch(units, keep_on_device=True)
        ms.append(sf.last_call_stats()["ms_total"])
    st = sf.last_call_stats()
    outs = sf.seed_and_filter_batch(units)
    exact = True
    for r in (0, 1):
        got = distinct_rows([o[1:] for u, o in zip(units, outs) if u[1] == r])
        want = distinct_rows([o[1:] for u, o in zip(chunked_units, chunked_outs) if u[1] == r])
        exact = exact and got.shape == want.shape and np.array_equal(got, want)
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        tuned = sf.autotune(units, cache_path=os.path.join(d, "tune.jsonl"), quick=True, repeats=1)
    return {"units": len(units), "extensions_per_step": st["num_hits"], "ms_per_step": min(ms),
            "value": st["num_hits"] / (min(ms) / 1000.0), "hsps_per_step": st["num_hsps"],
            "bit_exact_distinct_vs_250kbp_chunks": bool(exact), "autotune_quick": tuned}


def run_serving(sf, target: bytes, n_req: int, table: str, bursts: int = 3) -> dict:
    """Serving leg: capacity = median rate of `bursts` closed-loop bursts of
    the request set (after one untimed burst that grows the request-buffer
    pool and pinned output buffers), then Poisson arrivals at 0.5x, 1x and 2x
    of it; latency = submission -> HSP lists on the host."""
    reqs = serve_requests(target, n_req, seed=105)
    sf.serve_start(interval_size=INTERVAL, interval_overlap=OVERLAP, chunk_size=CHUNK, strands=3)
    try:
        alone = {}
        for k in range(4):  # a sample run alone, to compare with the same requests in the mix
            alone[k] = sf.serve_wait(sf.serve_submit(reqs[k]))[:2]
        for r in [sf.serve_submit(q) for q in reqs]:
            sf.serve_wait(r)
        caps = []
        for _ in range(bursts):
            ids = [sf.serve_submit(q) for q in reqs]
            st = [sf.serve_wait(r)[2] for r in ids]
            caps.append(len(reqs) / (max(x["done_s"] for x in st) - min(x["submit_s"] for x in st)))
        cap = float(statistics.median(caps))
        rates = []
        exact = True
        for load in (0.5, 1.0, 2.0):
            rng = np.random.default_rng(int(load * 100))
            gaps = rng.exponential(1.0 / (load * cap), size=len(reqs))
            ids = []
            t0 = time.perf_counter()
            t_next = 0.0
            for q, g in zip(reqs, gaps):
                t_next += g
                d = t_next - (time.perf_counter() - t0)
                if d > 0:
                    time.sleep(d)
                ids.append(sf.serve_submit(q))
            res = [sf.serve_wait(r) for r in ids]
            st = [x[2] for x in res]
            for k, (fw, rc) in alone.items():
                exact = exact and np.array_equal(res[k][0].view(np.uint32), fw.view(np.uint32)) and \
                    np.array_equal(res[k][1].view(np.uint32), rc.view(np.uint32))
            lat = np.array([x["done_s"] - x["submit_s"] for x in st]) * 1000.0
            wall = max(x["done_s"] for x in st) - min(x["submit_s"] for x in st)
            rates.append({"load": load, "offered_rps": load * cap, "p50_ms": float(np.percentile(lat, 50)),
                          "p99_ms": float(np.percentile(lat, 99)), "max_ms": float(lat.max()),
                          "extensions_per_s": sum(x["num_hits"] for x in st) / wall,
                          "hsps_per_s": sum(x["num_hsps"] for x in st) / wall,
                          "mean_passes_per_request": float(np.mean([x["num_passes"] for x in st]))})
    finally:
        sf.serve_stop()
    return {"workload": f"{n_req} requests per load, lengths log-uniform 10 kbp-20 Mbp (mean "
                        f"{np.mean([len(q) for q in reqs]) / 1e6:.2f} Mbp), 30% target blocks at 20% divergence, "
                        f"both strands, against the resident {table}",
            "capacity_rps": cap, "capacity_bursts_rps": caps, "loads": rates,
            "bit_exact_alone_vs_mix": bool(exact)}


def ref_gpu_baseline(sf, w, calls, n_units: int) -> dict:
    """Unranked: the reference's own SeedAndFilter (src/seed_filter.cu, compiled
    unmodified for sm_100a, oracle/ref_harness.cu) on the first n_units units
    of the workload, per-call wall time on this GPU, and whether its outputs
    equal ours call by call.  Inputs pass through oracle.ref_safe_texts, which
    changes no seed and no score (our results on them equal those on the
    original texts), and seeds the harness would refuse are dropped on both
    sides."""
    import oracle
    from segalign_b200 import host_revcomp, host_seeds

    if not oracle.ref_harness_available("plain"):
        return {"unavailable": "oracle/_ref/ref_seedfilter not built (needs the reference tree at build time)"}
    T, Q = oracle.ref_safe_texts(w.target, w.query)
    p = oracle.params()
    tk = oracle.ref_tail_keys(T, p)
    rct = host_revcomp(Q)
    sample = []
    for (_, rev, a, b) in calls[:n_units]:
        seeds = oracle.ref_filter_seeds(host_seeds(rct if rev else Q, a, b), tk, len(Q))
        if len(seeds):
            sample.append({"rev": rev, "seeds": seeds})
    t0 = time.perf_counter()
    ref = oracle.ref_seed_and_filter(sample, T, Q, timeout=900)
    harness_s = time.perf_counter() - t0
    exact = True
    for c, r in zip(sample, ref):
        got = sf.seed_and_filter(c["seeds"], bool(c["rev"]), 0)
        exact = exact and len(got) == len(r["segments"]) and \
            np.array_equal(got.view(np.uint32)[2:], r["segments"].view(np.uint32)[2:])
    secs = sum(r["seconds"] for r in ref)
    hits = sum(r["num_hits"] for r in ref)
    return {"value": hits / secs, "unit": UNIT, "calls": len(ref), "extensions": hits, "seconds": secs,
            "hsps": int(sum(r["num_hsps"] for r in ref)), "harness_wall_s": harness_s,
            "kind": "reference src/seed_filter.cu SeedAndFilter compiled for sm_100a, one call at a time, "
                    "per-call wall time (host vectors in and out)",
            "bit_exact_vs_ours": bool(exact)}


def allreduce_value(x: float, op: str, dist=None, device: str = "cuda") -> float:
    """One scalar reduced over the ranks ("max" or "sum"); the value itself on one rank."""
    if dist is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def job_figures(ms_step: float, hits: float, hsps: float, dist=None, device: str = "cuda") -> dict:
    """Whole-job figures of a step: every rank runs its share of the job, so
    the step lasts as long as the slowest rank and the work of all ranks adds
    up."""
    ms = allreduce_value(ms_step, "max", dist, device)
    h = allreduce_value(hits, "sum", dist, device)
    hs = allreduce_value(hsps, "sum", dist, device)
    return {"ms_per_step": ms, "extensions": h, "hsps": hs, "value": h / (ms / 1000.0),
            "hsps_per_s": hs / (ms / 1000.0)}


def make_workload(args, rank: int = 0, world: int = 1):
    """(workload, transition, description) of --workload for one rank of a job
    over `world` ranks.  The target is the same on every rank (replicated, as
    the reference replicates it to every GPU).  Weak scaling: the job's query is
    `world` blocks of the named size, drawn from that target, and rank r runs
    block r (block 0 is the one-GPU workload).  Strong scaling: the job is the
    named query and rank r runs its r-th contiguous slice."""
    from segalign_b200 import synth

    weak = getattr(args, "scaling", "weak") == "weak"
    block = rank if (weak and world > 1) else 0
    if args.workload == "large":
        w = synth.make(4, seed=104, scale=args.scale, block=block)
        q = w.query[: args.query_sample]
        desc = (f"large: 600 Mbp target (12 chr) x the first {len(q) / 1e6:.0f} Mbp of a 600 Mbp query, "
                "GC 41%, 45% repeats, 12of19 with one transition, HOXD70, xdrop 910, hspthresh 3000, entropy, "
                "both strands, 10 Mbp intervals + 50 kbp overlap, 250 kbp units")
        transition = True
    else:
        w = synth.make(2, seed=102, scale=args.scale, block=block)
        q = w.query
        desc = ("genome scale: 100 Mbp target (6 chr) x 108 Mbp query, GC 36%, 12of19, HOXD70, xdrop 910, "
                "hspthresh 3000, entropy, both strands, 10 Mbp intervals + 50 kbp overlap, 250 kbp units")
        transition = False
    if world > 1:
        if weak:
            desc += f"; job: {world} query blocks of this size against the one target, block r on rank r"
        else:
            a, b = len(q) * rank // world, len(q) * (rank + 1) // world
            q = q[a:b]
            desc += f"; job: this query split into {world} contiguous slices, slice r on rank r"
    return synth.Workload(w.target, q, w.target_chr, [(0, len(q))]), transition, desc


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    w, transition, desc = make_workload(args, 0)
    threads = os.cpu_count() or 1
    vals = []
    last = None
    for k in range(args.warmup + args.steps):
        r = cpu_sample(w, args.cpu_chunks, threads, transition)
        if k >= args.warmup:
            vals.append(r["hits"] / r["seconds"])
        last = r
    v = float(statistics.median(vals)) if vals else 0.0
    sample = (f"first {args.cpu_chunks} SeedAndFilter units (250 kbp, seeder order: interval 0 plus strand, then "
              f"minus) of the {args.workload} workload; {last['hits']} extensions per step")
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000.0 * last["seconds"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": desc, "sample_units": args.cpu_chunks},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "hsps_per_s": last["hsps"] / last["seconds"],
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# Our implementation
# ---------------------------------------------------------------------------
def timed_batch_steps(sf, units, steps: int, flush, barrier):
    """`steps` timed passes of the batched form, each from the resident query
    text to the HSP lists on the host: device seeding (per-position keys
    recomputed), lookup, extension, dedup, the records' copy to the host and
    their per-unit lists.  Returns per-step wall seconds, device milliseconds
    (CUDA events of the library's stream) and the last step's statistics."""
    import torch

    wall, dev, lane, warp, lk, dd = [], [], [], [], [], []
    outs = st = None
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        # CUDA events on the current stream bracket the step: the calls return
        # only once the HSP lists are on the host, so the end event is taken
        # after the whole step
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        sf.refresh_query_keys(0)
        outs = sf.seed_and_filter_batch(units)
        e1.record()
        e1.synchronize()
        wall.append(e0.elapsed_time(e1) / 1000.0)
        st = sf.last_call_stats()
        dev.append(st["ms_total"])
        lane.append(st["ms_extend_lane"])
        warp.append(st["ms_extend_warp"])
        lk.append(st["ms_lookup"])
        dd.append(st["ms_dedup"])
    barrier()
    mean = lambda x: sum(x) / len(x)  # noqa: E731
    return {"wall_s": wall, "dev_ms": mean(dev), "lane_ms": mean(lane), "warp_ms": mean(warp), "lookup_ms": mean(lk),
            "dedup_ms": mean(dd), "stats": st, "outs": outs}


def plain_device_ms(sf, w, calls) -> float:
    """Device time of the plain path: every unit as its own sa_seed_and_filter
    call, one at a time, summed over the units (CUDA events per call)."""
    from segalign_b200 import host_revcomp, host_seeds

    rct = host_revcomp(w.query)
    sf.set_timing(True)
    total = 0.0
    for (_, rev, a, b) in calls:
        seeds = host_seeds(rct if rev else w.query, a, b)
        if len(seeds):
            sf.seed_and_filter(seeds, bool(rev), 0)
            total += sf.last_call_stats()["ms_total"]
    return total


def run_ours(args):
    import torch

    from segalign_b200 import SeedFilter, build_sub_mat

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    def allreduce(x: float, op: str) -> float:
        return allreduce_value(x, op, dist)

    # one job over the ranks: the target replicated, the query in blocks
    # (weak scaling) or slices (strong scaling), no data exchanged between ranks
    w, transition, desc = make_workload(args, rank, world)
    sf = SeedFilter()
    sf.initialize_interface(1)
    sf.generate_shape_pos("12of19")
    os.environ.setdefault("SA_SLOTS_PER_GPU", "12")  # concurrent plain calls per GPU (e2e leg)
    sf.initialize_processor(transition, CHUNK, SEED_SIZE, build_sub_mat(910), 910, 3000, False)
    sf.send_ref_write_request(w.target)
    t = time.perf_counter()
    sf.generate_seed_pos_table(None, 1, SEED_SIZE, 12)
    torch.cuda.synchronize()
    table_ms = 1000 * (time.perf_counter() - t)
    sf.send_query_write_request(w.query, 0)
    calls = seeder_calls(len(w.query))
    plus = [c for c in calls if c[1] == 0]
    minus = [c for c in calls if c[1] == 1]
    units = plus + minus
    unit_of = {c: i for i, c in enumerate(units)}
    sf.set_timing(True)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")  # > 126 MB L2

    # ---- value: batched form, query text resident -> HSP lists on the host ----
    # the warm-up holds each step's lists while the next step runs, as the
    # timed loop does, so the library's output arrays reach their steady state
    held = None
    for _ in range(args.warmup):
        sf.refresh_query_keys(0)
        held = sf.seed_and_filter_batch(units)
    del held
    barrier()
    l0 = sf.kernel_launches()
    with ClockSampler(gpu_index(local)) as clk:
        tb = timed_batch_steps(sf, units, args.steps, flush, barrier)
    launches = sf.kernel_launches() - l0
    st = tb["stats"]
    outs = tb["outs"]
    hits, hsps, surv, tiles, nnz, longs = (st["num_hits"], st["num_hsps"], st["survivors"], st["tiles"],
                                           st["seeds_with_hits"], st["long_hits"])
    ms_step = 1000.0 * sum(tb["wall_s"]) / len(tb["wall_s"])
    job = job_figures(ms_step, float(hits), float(hsps), dist)
    ms_step_max, hits_all, hsps_all, value = job["ms_per_step"], job["extensions"], job["hsps"], job["value"]

    # roofline of the dominant kernel (lane-per-hit X-drop): algorithmic bytes
    # = 24 B per hit-bearing seed (E, lo, j, scope, unit) + 4 B per hit (pos)
    # + 24 B per 32-base tile scanned (2 sequences x 32 bases x 3 bits)
    # + 16 B per surviving HSP record
    lane_ms_avg = tb["lane_ms"]
    alg_bytes = 24.0 * nnz + 4.0 * hits + 24.0 * tiles + 16.0 * surv
    peak, peak_src = peaks()
    achieved = alg_bytes / (lane_ms_avg / 1000.0) / 1e9
    traffic, traffic_src = lane_traffic(hits, args.workload)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "traffic_source": traffic_src, "kernel": "sa_k_extend_lane",
                "peak_source": peak_src, "alg_bytes_per_launch": alg_bytes, "launch_ms": lane_ms_avg,
                "limit": lane_limit(args.workload)}

    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_step_max, "higher_is_better": True, "scaling": args.scaling, "vs_baseline": None,
        "dtype": "int32", "data": "synthetic",
        "config": {"workload": desc, "path": "batched: resident query text -> device seeding, lookup, X-drop, dedup "
                   "-> HSP lists on the host", "units": len(units), "target_bp": len(w.target),
                   "query_bp": len(w.query), "l2": "flushed between steps (512 MiB write)", "scale": args.scale,
                   "parallelism": (f"{world} ranks, one job: target replicated, query "
                                   f"{'blocks' if args.scaling == 'weak' else 'slices'} across ranks, "
                                   "no collective on the data path" if world > 1 else "1 GPU")},
        "hsps_per_s": hsps_all / (ms_step_max / 1000.0),
        "extensions_per_step": hits_all, "hsps_per_step": hsps_all,
        "device_ms_per_step": tb["dev_ms"],
        "phase_ms": {"lookup": tb["lookup_ms"], "extend_lane": lane_ms_avg, "extend_warp": tb["warp_ms"],
                     "dedup": tb["dedup_ms"], "device_total": tb["dev_ms"], "wall_per_step": ms_step},
        "table_build_ms": table_ms,
        "roofline": roofline,
        "gpu_launches": launches,
        "clocks": clk.summary(),
        "counts": {"survivors": surv, "long_hits": longs, "tiles": tiles, "seeds_with_hits": nnz},
    }

    # ---- e2e: reference-facing C ABI (host seeds in, host HSP lists out) ----
    if not args.no_e2e:
        k_e2e = args.e2e_steps or max(1, min(args.steps, 3))
        sf.set_timing(False)
        e2e_threads = min(16, os.cpu_count() or 8)
        sf.seeder_run(w.query, buffer=0, strand=3, num_threads=e2e_threads, interval_size=INTERVAL, chunk_size=CHUNK,
                      interval_overlap=OVERLAP, transition=transition)
        barrier()
        t0 = time.perf_counter()
        for _ in range(k_e2e):
            fw, rc, sst = sf.seeder_run(w.query, buffer=0, strand=3, num_threads=e2e_threads,
                                        interval_size=INTERVAL, chunk_size=CHUNK, interval_overlap=OVERLAP,
                                        transition=transition)
        barrier()
        e2e_s = (time.perf_counter() - t0) / k_e2e
        e2e_s_max = allreduce(e2e_s, "max")
        e2e_hits = allreduce(float(sst["num_hits"]), "sum")
        # per call: seed words + call descriptor (32 B) + unit (32 B) + scope flags (1 KiB) up;
        # counters (128 B) + header and HSP records (16 B each) down
        h2d = sst["num_seeds"] * 8 + sst["num_calls"] * (32 + 32 + 1024)
        d2h = (sst["num_hsps"] + sst["num_calls"]) * 16 + sst["num_calls"] * 128
        out["e2e"] = {"value": e2e_hits / e2e_s_max, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                      "d2h_bytes_per_step": int(d2h), "path": f"sa_seed_and_filter per 250 kbp unit from "
                      f"{e2e_threads} host threads (C++ seeder), host wall time", "steps": k_e2e}
        # batched with host buffers: query text up, HSP lists down (one untimed
        # step first: it sizes the pinned output buffer)
        sf.set_timing(True)
        sf.send_query_write_request(w.query, 1)
        sf.seed_and_filter_batch([(1, r, a, b) for (_, r, a, b) in units])
        barrier()
        t0 = time.perf_counter()
        outs1 = None
        t_write = t_call = 0.0
        for _ in range(k_e2e):
            t1 = time.perf_counter()
            sf.send_query_write_request(w.query, 1)
            t2 = time.perf_counter()
            outs1 = sf.seed_and_filter_batch([(1, r, a, b) for (_, r, a, b) in units])
            t_write, t_call = t_write + t2 - t1, t_call + time.perf_counter() - t2
        barrier()
        eb_s = allreduce((time.perf_counter() - t0) / k_e2e, "max")
        out["e2e_batched"] = {"value": e2e_hits / eb_s, "unit": UNIT, "h2d_bytes_per_step": len(w.query),
                              "d2h_bytes_per_step": int(sum(len(o) for o in outs1) * 16),
                              "query_write_s": t_write / k_e2e, "batch_call_s": t_call / k_e2e}
        sf.clear_query(1)
        # bit-exact: batched units == plain per-call results (concatenated per strand)
        bf = np.concatenate([o[1:] for o in outs[: len(plus)]]) if plus else np.zeros(0)
        br = np.concatenate([o[1:] for o in outs[len(plus):]]) if minus else np.zeros(0)
        out["bit_exact_batched_vs_plain"] = bool(
            len(bf) == len(fw) and len(br) == len(rc) and np.array_equal(bf.view(np.uint32), fw.view(np.uint32))
            and np.array_equal(br.view(np.uint32), rc.view(np.uint32)))
        # like for like: host buffers on both sides, and device time on both sides
        dp_ms = plain_device_ms(sf, w, units) if world == 1 else None
        out["batched_vs_plain"] = {
            "e2e_batched_over_e2e": out["e2e_batched"]["value"] / out["e2e"]["value"],
            "device_plain_ms": dp_ms, "device_batched_ms": tb["dev_ms"],
            "device_plain_over_device_batched": (dp_ms / tb["dev_ms"]) if dp_ms else None,
            "note": "e2e: host buffers on both sides; device: the units one call at a time (events, summed) "
                    "against one batched pass"}

    # ---- batched form over uneven windows, distinct HSPs vs the chunked run ----
    if not args.no_e2e:
        saved = sf.get_tuning()
        out["batched_uneven"] = run_uneven(sf, len(w.query), outs, units)
        sf.set_tuning(**saved)

    # ---- serving form (one GPU): Poisson request stream over the resident table ----
    if world == 1 and not args.no_serve:
        sf.set_timing(False)
        n_req = args.serve_requests or (args.large_serve_requests if args.workload == "large" else 200)
        table = ("600 Mbp target table (transitions on)" if args.workload == "large"
                 else "100 Mbp genome-scale target table")
        out["serving"] = run_serving(sf, w.target, n_req, table)

    # ---- unranked: the reference's own kernels on a sample of the same units ----
    if world == 1 and rank == 0 and not args.no_ref_gpu and args.workload == "genome":
        try:
            out["ref_gpu_baseline"] = ref_gpu_baseline(sf, w, calls, args.ref_gpu_units)
        except Exception as e:  # the reference harness is a checker: report, do not fail the bench
            out["ref_gpu_baseline"] = {"unavailable": f"{type(e).__name__}: {str(e)[:300]}"}

    # ---- CPU baseline on a bounded sample (rank 0, one GPU only) ----
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        r = cpu_sample(w, args.cpu_chunks, threads, transition)
        cpu_v = r["hits"] / r["seconds"]
        out["cpu_baseline"] = {"value": cpu_v, "unit": UNIT, "cores": threads, "kind": "port",
                               "sample": f"first {args.cpu_chunks} 250 kbp units of the same workload "
                                         f"({r['hits']} extensions, {r['seconds']:.1f} s)"}
        # the sampled calls (seeder order), GPU batched units vs CPU port, bit-exact
        samp = calls[: args.cpu_chunks]
        gf = [outs[unit_of[c]][1:] for c in samp if c[1] == 0]
        gr = [outs[unit_of[c]][1:] for c in samp if c[1] == 1]
        gf = np.concatenate(gf) if gf else np.zeros(0, dtype=r["fw"].dtype)
        gr = np.concatenate(gr) if gr else np.zeros(0, dtype=r["rc"].dtype)
        out["bit_exact_vs_cpu_sample"] = bool(
            len(gf) == len(r["fw"]) and len(gr) == len(r["rc"])
            and np.array_equal(gf.view(np.uint32), r["fw"].view(np.uint32))
            and np.array_equal(gr.view(np.uint32), r["rc"].view(np.uint32)))

    # ---- whole files: the same workload as FASTA through sa_align_fasta (one GPU) ----
    if world == 1 and args.workload == "genome" and not args.no_fasta:
        out["fasta"] = run_fasta(sf, w, None if args.no_e2e else sst)

    # ---- the 600 Mbp legs (one GPU): config 4 batched and plain, config 5 serving, repeat masker ----
    if world == 1 and args.workload == "genome" and not args.no_large:
        del w, outs
        out["large"] = run_large(sf, args, flush, barrier)
    elif args.workload == "large" and args.rm_intervals and world == 1:
        out["rm_self_alignment"] = run_rm(sf, w.target, args.rm_intervals, transition)

    if rank == 0:
        print(json.dumps(out), flush=True)
    sf.shutdown_processor()
    if dist:
        dist.destroy_process_group()
    return 0


def run_fasta(sf, w, e2e_stats) -> dict:
    """Whole-file leg: the workload written as FASTA (one record per target
    chromosome, the query as one record) and run through sa_align_fasta, the
    path of the reference's main.cpp minus lastz: parse, '&'-joined blocks,
    target upload and seed-table build, double-buffered query upload, the C++
    seeder over plain calls on 16 host threads, and the segment writer on the
    GPU into a segments file.  Host wall time of the one call.  Its hits and
    HSPs equal the e2e leg's (same text, intervals and chunks)."""
    import shutil
    import tempfile

    d = tempfile.mkdtemp(prefix="sa_fasta_")
    try:
        tp, qp, sp = (os.path.join(d, n) for n in ("target.fa", "query.fa", "out.segments"))
        for path, text, chrs, tag in ((tp, w.target, w.target_chr, b"chr"), (qp, w.query, w.query_chr, b"q")):
            with open(path, "wb") as f:
                for i, (a, n) in enumerate(chrs):
                    f.write(b">%s%d\n" % (tag, i + 1))
                    f.write(text[a:a + n])
                    f.write(b"\n")
        threads = min(16, os.cpu_count() or 8)
        t0 = time.perf_counter()
        st = sf.align_fasta(tp, qp, segments_path=sp, interval_size=INTERVAL, interval_overlap=OVERLAP,
                            chunk_size=CHUNK, num_threads=threads)
        dt = time.perf_counter() - t0
        res = {"workload": f"the genome-scale workload as FASTA files ({len(w.target_chr)} target records, "
                           f"{len(w.query_chr)} query record) to a lastz --segments file, {threads} host threads",
               "seconds": dt, "read_s": st["read_seconds"], "table_s": st["table_seconds"],
               "query_write_s": st["query_write_seconds"], "calls_s": st["calls_seconds"],
               "output_s": st["output_seconds"], "hits": st["num_hits"], "hsps": st["num_hsps"],
               "extensions_per_s": st["num_hits"] / dt, "segments_bytes": os.path.getsize(sp),
               "fasta_bytes": os.path.getsize(tp) + os.path.getsize(qp)}
        if e2e_stats is not None:
            res["same_hits_and_hsps_as_e2e"] = bool(st["num_hits"] == e2e_stats["num_hits"]
                                                    and st["num_hsps"] == e2e_stats["num_hsps"])
        return res
    finally:
        shutil.rmtree(d, ignore_errors=True)


def run_rm(sf, target: bytes, n_intervals: int, transition: bool) -> dict:
    """Repeat-masker self-alignment of the 600 Mbp target: the first n_intervals
    10 Mbp intervals against their neighbour windows (it re-sends the target)."""
    sf.set_rm_exclude_diagonal(True)
    try:
        runs, rst = sf.rm_seeder_run(target, strand=3, num_threads=16, max_intervals=n_intervals,
                                     transition=transition)
    finally:
        sf.set_rm_exclude_diagonal(False)
    return {"workload": f"first {rst['num_intervals']} of the 10 Mbp intervals of the 600 Mbp target against "
                        "their neighbour windows (proportion 0.2), both strands, transitions, diagonal excluded, M 1",
            "seconds": rst["seconds"], "hits": rst["num_hits"], "hits_per_s": rst["num_hits"] / rst["seconds"],
            "hsps": rst["num_hsps"], "calls": rst["num_calls"], "runs": int(len(runs)),
            "covered_bases": int(runs["len"].sum()) if len(runs) else 0}


def run_large(sf, args, flush, barrier) -> dict:
    """The 600 Mbp target (12 chr, GC 41%, 45% repeats) with transitions: the
    batched form over a query sample (value as for the genome workload), the
    plain C-ABI path on the same units, the serving form on that resident
    table, and the repeat-masker self-alignment of the target."""
    from segalign_b200 import build_sub_mat, synth

    t0 = time.perf_counter()
    w = synth.make(4, seed=104, scale=args.scale)
    q = w.query[: args.query_sample]
    gen_s = time.perf_counter() - t0
    sf.initialize_processor(True, CHUNK, SEED_SIZE, build_sub_mat(910), 910, 3000, False)
    sf.send_ref_write_request(w.target)
    t = time.perf_counter()
    sf.generate_seed_pos_table(None, 1, SEED_SIZE, 12)
    barrier()
    table_ms = 1000 * (time.perf_counter() - t)
    sf.send_query_write_request(q, 0)
    calls = seeder_calls(len(q))
    units = [c for c in calls if c[1] == 0] + [c for c in calls if c[1] == 1]
    sf.set_timing(True)
    sf.refresh_query_keys(0)
    sf.seed_and_filter_batch(units)  # warm-up
    barrier()
    tb = timed_batch_steps(sf, units, 2, flush, barrier)
    st = tb["stats"]
    wall = sum(tb["wall_s"]) / len(tb["wall_s"])
    alg = 24.0 * st["seeds_with_hits"] + 4.0 * st["num_hits"] + 24.0 * st["tiles"] + 16.0 * st["survivors"]
    peak, _ = peaks()
    res = {"workload": f"600 Mbp target (12 chr) x the first {len(q) / 1e6:.0f} Mbp of a 600 Mbp query, GC 41%, "
                       "45% repeats, 12of19 with one transition (13 seed words per position), both strands, "
                       f"{len(units)} units of 250 kbp", "generate_s": gen_s, "table_build_ms": table_ms,
           "value": st["num_hits"] / wall, "unit": UNIT, "ms_per_step": 1000 * wall,
           "device_ms_per_step": tb["dev_ms"], "extensions_per_step": st["num_hits"], "hsps_per_step": st["num_hsps"],
           "phase_ms": {"lookup": tb["lookup_ms"], "extend_lane": tb["lane_ms"], "extend_warp": tb["warp_ms"],
                        "dedup": tb["dedup_ms"]},
           "roofline": {"kernel": "sa_k_extend_lane", "achieved": alg / (tb["lane_ms"] / 1000) / 1e9, "peak": peak,
                        "frac": alg / (tb["lane_ms"] / 1000) / 1e9 / peak, "unit": "GB/s",
                        "traffic": lane_traffic(st["num_hits"], "large")[0]}}
    outs = tb["outs"]
    # plain path with host buffers on the same units (seeds with transitions on the host)
    sf.set_timing(False)
    fw, rc, sst = sf.seeder_run(q, buffer=0, strand=3, num_threads=16, interval_size=INTERVAL, chunk_size=CHUNK,
                                interval_overlap=OVERLAP, transition=True)
    barrier()
    t0 = time.perf_counter()
    fw, rc, sst = sf.seeder_run(q, buffer=0, strand=3, num_threads=16, interval_size=INTERVAL, chunk_size=CHUNK,
                                interval_overlap=OVERLAP, transition=True)
    barrier()
    e2e_s = time.perf_counter() - t0
    nplus = sum(1 for c in calls if c[1] == 0)
    bf = np.concatenate([o[1:] for o in outs[:nplus]])
    br = np.concatenate([o[1:] for o in outs[nplus:]])
    res["e2e"] = {"value": sst["num_hits"] / e2e_s, "unit": UNIT, "seconds": e2e_s,
                  "h2d_bytes_per_step": int(sst["num_seeds"] * 8), "d2h_bytes_per_step": int(
                      (sst["num_hsps"] + sst["num_calls"]) * 16),
                  "path": "sa_seed_and_filter per 250 kbp unit from 16 host threads (C++ seeder with transitions)"}
    res["bit_exact_batched_vs_plain"] = bool(
        len(bf) == len(fw) and len(br) == len(rc) and np.array_equal(bf.view(np.uint32), fw.view(np.uint32))
        and np.array_equal(br.view(np.uint32), rc.view(np.uint32)))
    # CPU port on a bounded sample of the same units, bit-exact against the batched units
    if args.large_cpu_units:
        pw = synth.Workload(w.target, q, w.target_chr, w.query_chr)
        r = cpu_sample(pw, args.large_cpu_units, os.cpu_count() or 1, True)
        samp = calls[:args.large_cpu_units]
        unit_of = {c: i for i, c in enumerate(units)}
        gf = [outs[unit_of[c]][1:] for c in samp if c[1] == 0]
        gr = [outs[unit_of[c]][1:] for c in samp if c[1] == 1]
        gf = np.concatenate(gf) if gf else np.zeros(0, dtype=r["fw"].dtype)
        gr = np.concatenate(gr) if gr else np.zeros(0, dtype=r["rc"].dtype)
        res["cpu_sample"] = {"value": r["hits"] / r["seconds"], "units": args.large_cpu_units, "extensions": r["hits"],
                             "bit_exact": bool(len(gf) == len(r["fw"]) and len(gr) == len(r["rc"]) and
                                               np.array_equal(gf.view(np.uint32), r["fw"].view(np.uint32)) and
                                               np.array_equal(gr.view(np.uint32), r["rc"].view(np.uint32)))}
        _TABLES.clear()
    del outs
    if not args.no_serve:
        res["serving"] = run_serving(sf, w.target, args.large_serve_requests,
                                     "600 Mbp target table (transitions on)")
    if args.rm_intervals:
        res["rm_self_alignment"] = run_rm(sf, w.target, args.rm_intervals, True)
    return res


def main():
    args = parse_args()
    if args.cpu_chunks is None:
        args.cpu_chunks = 2 if args.workload == "large" else 64
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
