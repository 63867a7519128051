"""Golden fixtures (tests/golden/, made by make_golden.py): the oracle must
reproduce them on CPU, and the GPU path must reproduce them through the C ABI."""
import json
import os

import numpy as np
import pytest

import oracle

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load():
    arr = np.load(os.path.join(GOLD, "small_calls.npz"))
    meta = json.load(open(os.path.join(GOLD, "small_calls.json")))
    return arr, meta


def kat_cases():
    return json.load(open(os.path.join(GOLD, "kat_cases.json")))


def test_oracle_reproduces_kat_fixtures(built):
    for c in kat_cases():
        p = oracle.params(**c["params"])
        r = oracle.extend_hit(p, oracle.encode(c["R"].encode()), oracle.encode(c["Q"].encode()), c["ref_loc"],
                              c["query_loc"])
        assert {k: r[k] for k in c["expect"]} == c["expect"], c


def test_oracle_reproduces_call_fixtures(built):
    arr, meta = load()
    T, Qt = arr["target"].tobytes(), arr["query"].tobytes()
    p = oracle.params()
    idx, pos = oracle.build_table(T, p)
    R = oracle.encode(T)
    for c in meta["calls"]:
        rm = c["key"].startswith("rm")
        if rm:
            text = oracle.revcomp_text(T) if c["rev"] else T
            qc = oracle.rc_codes(R) if c["rev"] else R
        else:
            text = oracle.revcomp_text(Qt) if c["rev"] else Qt
            qc = oracle.encode_rc(Qt) if c["rev"] else oracle.encode(Qt)
        seeds = oracle.chunk_seeds(text, c["j0"], c["j1"], p)
        assert len(seeds) == c["num_seeds"]
        segs, st = oracle.seed_and_filter(p, R, qc, idx, pos, seeds, c["rev"], 1 if rm else 0,
                                          c.get("rm_ref_start", 0), c.get("rm_ref_end", 0))
        assert st["num_hits"] == c["num_hits"]
        assert np.array_equal(segs.view(np.uint32).reshape(-1, 4), arr[c["key"] + "_out"]), c["key"]


@pytest.mark.gpu
def test_gpu_reproduces_call_fixtures(built):
    from segalign_b200 import SeedFilter, build_sub_mat, host_revcomp, host_seeds

    arr, meta = load()
    T, Qt = arr["target"].tobytes(), arr["query"].tobytes()
    sf = SeedFilter()
    sf.initialize_interface(1)
    sf.generate_shape_pos("12of19")
    sf.initialize_processor(False, meta["chunk"], 19, build_sub_mat(910), 910, 3000, False)
    sf.send_ref_write_request(T)
    sf.generate_seed_pos_table(None, 1, 19, 12)
    sf.send_query_write_request(Qt, 0)
    sf.rm_send_query_write_request()
    for c in meta["calls"]:
        rm = c["key"].startswith("rm")
        src = T if rm else Qt
        text = host_revcomp(src) if c["rev"] else src
        seeds = host_seeds(text, c["j0"], c["j1"])
        if rm:
            got = sf.rm_seed_and_filter(seeds, bool(c["rev"]), c["rm_ref_start"], c["rm_ref_end"])
        else:
            got = sf.seed_and_filter(seeds, bool(c["rev"]), 0)
        assert np.array_equal(got.view(np.uint32).reshape(-1, 4), arr[c["key"] + "_out"]), c["key"]


@pytest.mark.gpu
def test_gpu_kat_hits_through_crafted_tables(built):
    """Each fixture hit is driven through the GPU as the only hit of a call:
    a one-entry table bucket (key 0) at ref_loc - 19 and one seed at query_loc - 19."""
    from segalign_b200 import SeedFilter, build_sub_mat

    sf = SeedFilter()
    for c in kat_cases():
        pr = c["params"]
        R, Q = c["R"].encode(), c["Q"].encode()
        rl, ql = c["ref_loc"], c["query_loc"]
        if rl + 19 > len(R) + 19 or rl - 19 + 19 > len(R):
            continue
        sf.initialize_interface(1)
        sf.generate_shape_pos("12of19")
        sf.initialize_processor(False, 1000, 19, build_sub_mat(pr["xdrop"]), pr["xdrop"], pr["hspthresh"],
                                pr["noentropy"])
        sf.send_ref_write_request(R)
        index = np.ones(1 << 24, dtype=np.uint32)
        sf.send_seed_pos_table(index, np.array([rl - 19], dtype=np.uint32))
        sf.send_query_write_request(Q, 0)
        got = sf.seed_and_filter(np.array([ql - 19], dtype=np.uint64), False, 0)
        e = c["expect"]
        assert int(got[0]["score"]) == 1
        if e["keep"]:
            rec = tuple(int(x) for x in got[1])
            assert rec == (rl - e["left_pos"], ql - e["left_pos"], e["right_pos"] + e["left_pos"], e["score"]), c
        else:
            assert len(got) == 1, c
