"""GPU test of the repeat-masker self-alignment driver (sa_rm_seeder_run): on
a repeat-rich 1.8 Mbp sequence cut into two blocks, its coverage runs must
equal the oracle pipeline's, committed in tests/golden/rm_runs.npz by
tests/golden/make_golden.py (the oracle's block/interval plan, rm
SeedAndFilter per chunk and strand, and uint8 coverage runs)."""
import json
import os

import numpy as np
import pytest

import oracle
from segalign_b200 import SeedFilter, build_sub_mat, synth

pytestmark = pytest.mark.gpu

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def fixture(built):
    with open(os.path.join(HERE, "rm_runs.json")) as f:
        meta = json.load(f)
    runs = np.load(os.path.join(HERE, "rm_runs.npz"))
    seq = synth.make(4, seed=meta["seed"], scale=meta["scale"]).target
    assert len(seq) == meta["seq_len"]
    return meta, runs, seq


@pytest.mark.parametrize("M,exclude", [(1, True), (2, False)])
def test_rm_seeder_matches_oracle(fixture, M, exclude):
    meta, runs, seq = fixture
    want = runs[f"M{M}_exclude{int(exclude)}"]
    sf = SeedFilter()
    sf.initialize_interface(1)
    sf.generate_shape_pos("12of19")
    sf.initialize_processor(False, 250_000, 19, build_sub_mat(910), 910, 3000, False)
    sf.set_rm_exclude_diagonal(exclude)
    try:
        got, st = sf.rm_seeder_run(seq, lastz_interval_size=meta["interval_size"], seq_block_size=meta["block_size"],
                                   prop=meta["prop"], M=M, chunk_size=meta["chunk"], strand=3, num_threads=4)
    finally:
        sf.set_rm_exclude_diagonal(False)
    plan = oracle.rm_plan(len(seq), meta["interval_size"], meta["block_size"], meta["prop"])
    assert st["num_blocks"] == 2 and st["num_intervals"] == len(plan)
    assert len(want) > 10
    g = np.stack([got["block"], got["interval"], got["query_start"], got["len"]], axis=1).astype(np.uint32)
    assert g.shape == want.shape and np.array_equal(g, want)
