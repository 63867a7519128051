"""The library's multi-GPU dispatch, on the CPU with a faked device count.

sa_seed_and_filter takes a slot (stream + workspace) from a pool shared by all
initialised GPUs, as the reference's SeedAndFilter takes a GPU from its pool
(src/seed_filter.cu:667-674, :748-753).  The slot policy lives in
segalign_b200/csrc/sa_slot_pool.h; tests/cpp/slot_pool_test.cpp drives it with
several fake devices and many caller threads: no slot is held twice, every
device serves calls, the first G concurrent callers land on G different
devices, and no device takes a further slot while a less-loaded one has a free
slot."""
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("pool") / "slot_pool_test")
    r = subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-I", os.path.join(ROOT, "segalign_b200", "csrc"),
                        "-o", out, os.path.join(HERE, "cpp", "slot_pool_test.cpp")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


@pytest.mark.parametrize("n_dev,per_dev,threads", [(1, 12, 16), (2, 12, 16), (4, 3, 16), (8, 2, 32), (3, 5, 7)])
def test_slot_pool_spreads_calls_over_devices(exe, n_dev, per_dev, threads):
    r = subprocess.run([exe, str(n_dev), str(per_dev), str(threads), "300"], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0 and r.stdout.startswith("ok"), r.stdout + r.stderr
    served = [int(x) for x in r.stdout.split()[1:]]
    assert len(served) == n_dev and all(s > 0 for s in served)
