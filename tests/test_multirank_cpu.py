"""The N>1 path of bench.py on CPU: two gloo ranks (127.0.0.1) reduce their
per-rank step figures the way the GPU ranks do over NCCL (step time = the
slowest rank, work = the sum), and the ranks run one job: the same target on
every rank, and the query in blocks (weak scaling: a block of the named size
per rank) or in slices of the one query (strong scaling), with no data
exchanged between ranks."""
import os
import socket
import sys
import zlib

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out_dir: str):
    import argparse

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        fig = bench.job_figures(100.0 + 50.0 * rank, 1000.0 * (rank + 1), 10.0 * (rank + 1), dist, device="cpu")
        weak, _, _ = bench.make_workload(argparse.Namespace(workload="genome", scale=0.002, scaling="weak"),
                                         rank, world)
        strong, _, _ = bench.make_workload(argparse.Namespace(workload="genome", scale=0.002, scaling="strong"),
                                           rank, world)
        with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
            f.write(f"{fig['ms_per_step']} {fig['extensions']} {fig['hsps']} {fig['value']} {len(weak.target)} "
                    f"{zlib.crc32(weak.target)} {len(weak.query)} {zlib.crc32(weak.query)} "
                    f"{zlib.crc32(strong.target)}\n")
        with open(os.path.join(out_dir, f"slice{rank}.bin"), "wb") as f:
            f.write(strong.query)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_like_the_gpu_ranks(tmp_path, built):
    import torch.multiprocessing as mp

    port = _free_port()
    mp.spawn(_rank, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    rows = [open(tmp_path / f"rank{r}.txt").read().split() for r in range(2)]
    for r in rows:
        ms, ext, hsps, value = (float(x) for x in r[:4])
        assert ms == 150.0 and ext == 3000.0 and hsps == 30.0
        assert value == pytest.approx(3000.0 / 0.15)
    assert rows[0][4:6] == rows[1][4:6]  # one target on every rank
    assert rows[0][8] == rows[1][8] == rows[0][5]  # the same target in both modes
    assert rows[0][6] == rows[1][6] and rows[0][7] != rows[1][7]  # weak: query blocks of one size, distinct
    import argparse

    sys.path.insert(0, ROOT)
    import bench

    one, _, _ = bench.make_workload(argparse.Namespace(workload="genome", scale=0.002, scaling="weak"))
    assert zlib.crc32(one.query) == int(rows[0][7])  # block 0 is the one-GPU workload
    halves = (tmp_path / "slice0.bin").read_bytes() + (tmp_path / "slice1.bin").read_bytes()
    assert halves == one.query  # strong: the slices partition the one query
