"""The N>1 path of bench.py on CPU: two gloo ranks (127.0.0.1) reduce their
per-rank step figures the way the GPU ranks do over NCCL (step time = the
slowest rank, work = the sum), and each rank gets its own genome pair of the
same shape (weak scaling, no data exchanged between ranks)."""
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
        w, transition, _ = bench.make_workload(argparse.Namespace(workload="genome", scale=0.002), rank)
        with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
            f.write(f"{fig['ms_per_step']} {fig['extensions']} {fig['hsps']} {fig['value']} {len(w.target)} "
                    f"{zlib.crc32(w.target)}\n")
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
    assert rows[0][4] == rows[1][4]  # same shape
    assert rows[0][5] != rows[1][5]  # different genomes (seeds 102 and 1102)
