"""Known-answer tests of the oracle's X-drop, entropy and dedup semantics.

Each expected value is derived by hand from the reference source
(src/seed_filter.cu:204-624 find_hsps; :47-80, :728-732 sort/unique;
repeat_masker_src/seed_filter.cu:45-107 diagonal comparators).
"""
import math

import numpy as np
import pytest

import oracle

HOXD70 = [[91, -114, -31, -123], [-114, 100, -125, -31], [-31, -125, 100, -114], [-123, -31, -114, 91]]


def pm10_params(xdrop, hspthresh=30, noentropy=True):
    """+10 match / -10 mismatch on ACGT, the rest of the table as the reference builds it."""
    p = oracle.params(xdrop=xdrop, hspthresh=hspthresh, noentropy=noentropy)
    for r in range(4):
        for q in range(4):
            p.sub_mat[r * 8 + q] = 10 if r == q else -10
    return p


def codes(s: str) -> np.ndarray:
    return oracle.encode(s.encode())


def test_scoring_table_default(built):
    m = oracle.sub_mat(910).reshape(8, 8)
    assert m[:4, :4].tolist() == HOXD70
    assert (m[4, :5] == -1000).all() and (m[:5, 4] == -1000).all()          # lowercase
    assert (m[5, :6] == -1000).all() and (m[:6, 5] == -1000).all()          # N
    assert (m[6, :4] == -100).all() and m[6, 6] == -100 and m[6, 4] == -1000  # other IUPAC
    assert (m[7, :] == -9100).all() and (m[:, 7] == -9100).all()            # separator '&'


def test_scoring_table_ambiguous_n(built):
    m = oracle.sub_mat(910, "n").reshape(8, 8)
    assert (m[5, :5] == 0).all() and m[5, 5] == 0 and m[6, 6] == -100
    m = oracle.sub_mat(910, "iupac").reshape(8, 8)
    assert (m[6, :6] == 0).all() and m[6, 6] == 0
    m = oracle.sub_mat(910, "x,5,7").reshape(8, 8)
    assert m[6, 6] == -100 and m[5, 5] == -1000  # field 'x': only reward/penalty values change
    m = oracle.sub_mat(910, "n,5,7").reshape(8, 8)
    assert m[5, 5] == 5 and m[5, 0] == -7


def test_pure_match_run_to_both_edges(built):
    s = "ACGT" * 50
    p = oracle.params()
    r = oracle.extend_hit(p, codes(s), codes(s), 100, 100)
    # right: offsets 0..99 (edge at 100), 25 * (91+100+100+91); left: offsets 1..100
    assert (r["right_best"], r["right_pos"]) == (9550, 99)
    assert (r["left_best"], r["left_pos"]) == (9550, 100)
    assert r["total"] == 19100 and r["keep"] == 1 and r["score"] == 19100 and r["entropy_branch"] == 0
    # lane-31 edge test: offset 100 lies in right tile 3; left edge offset 101 in tile 3
    assert (r["tiles_right"], r["tiles_left"]) == (4, 4)


def test_no_positive_score_gives_rpos_minus_one(built):
    R = codes("A" * 64)
    Q = codes("T" * 64)
    r = oracle.extend_hit(oracle.params(), R, Q, 32, 32)
    # A/T = -123: best stays 0; 0 - S > 910 first at the 8th base (984)
    assert (r["right_best"], r["right_pos"], r["left_best"], r["left_pos"]) == (0, -1, 0, 0)
    assert r["keep"] == 0 and r["tiles_right"] == 1 and r["tiles_left"] == 1


def test_first_maximum_wins_ties(built):
    # scores +10 -10 +10 then -10s: S = 10, 0, 10, 0, -10, ...; xdrop 25 stops at S=-20 (M-S=30)
    R = codes("AAAAAAAAAAAA" + "ACAAAAAAA")
    Q = codes("AAAAAAAAAAAA" + "AAACCCCCC")
    p = pm10_params(xdrop=25)
    r = oracle.extend_hit(p, R, Q, 12, 12)
    assert (r["right_best"], r["right_pos"]) == (10, 0)


def test_xdrop_is_strict(built):
    # S: 10, 0, -10 (M-S = 20, not > 20), then five +10s up to 40 at o=7, then -10s
    R = codes("A" * 10 + "A" + "CC" + "AAAAA" + "C" * 10)
    Q = codes("A" * 10 + "A" + "AA" + "AAAAA" + "A" * 10)
    r = oracle.extend_hit(pm10_params(xdrop=20), R, Q, 10, 10)
    assert (r["right_best"], r["right_pos"]) == (40, 7)
    r = oracle.extend_hit(pm10_params(xdrop=19), R, Q, 10, 10)
    assert (r["right_best"], r["right_pos"]) == (10, 0)


@pytest.mark.parametrize("stopper", ["N", "&", "a"])
def test_n_separator_and_lowercase_stop_extension(built, stopper):
    s = "ACGT" * 10
    R = codes(s + stopper + s)
    Q = codes(s + "A" + s)
    r = oracle.extend_hit(oracle.params(), R, Q, 20, 20)
    # right covers offsets 0..19 (up to the stopper at position 40)
    assert r["right_pos"] == 19 and r["right_best"] == 5 * 382


def test_entropy_branch_float_log4(built):
    # 40-base ACGT run flanked by A/T mismatches: total 3820 in [3000, 9000],
    # counts 10/10/10/10 -> E = ln(1/4) / (double)logf(4.0f) = 0.99999999725...
    R = codes("A" * 50 + "ACGT" * 10 + "A" * 50)
    Q = codes("T" * 50 + "ACGT" * 10 + "T" * 50)
    r = oracle.extend_hit(oracle.params(), R, Q, 70, 70)
    assert r["total"] == 3820 and r["entropy_branch"] == 1
    e = -(4 * math.fma(0.25, math.log(0.25), 0.0) if False else math.log(0.25)) / float(np.float32(math.log(4.0)))
    assert abs(r["entropy"] - e) < 1e-15 and r["entropy"] < 1.0
    assert r["keep"] == 1 and r["score"] == 3819


def test_low_complexity_is_filtered(built):
    R = codes("C" * 50 + "A" * 40 + "C" * 50)
    Q = codes("G" * 50 + "A" * 40 + "G" * 50)
    r = oracle.extend_hit(oracle.params(), R, Q, 70, 70)
    assert r["total"] == 3640 and r["entropy_branch"] == 1
    assert r["entropy"] == 0.0 and r["keep"] == 0  # -(1 * ln 1) = 0


def test_noentropy_keeps_score(built):
    R = codes("C" * 50 + "A" * 40 + "C" * 50)
    Q = codes("G" * 50 + "A" * 40 + "G" * 50)
    r = oracle.extend_hit(oracle.params(noentropy=True), R, Q, 70, 70)
    assert r["keep"] == 1 and r["score"] == 3640


def test_dedup_sort_order_and_predecessor_unique(built):
    """A call whose hits all land on one segment yields it once; hspComp order across segments."""
    s = "ACGT" * 30
    T = ("C" * 40 + s + "C" * 40).encode()
    Q = ("G" * 40 + s + "G" * 40).encode()
    p = oracle.params()
    idx, pos = oracle.build_table(T, p)
    seeds = oracle.chunk_seeds(Q, 0, len(Q) - 19, p)
    out, st = oracle.seed_and_filter(p, oracle.encode(T), oracle.encode(Q), idx, pos, seeds, False)
    # every hit on the main diagonal extends to the full 120-base run
    assert st["num_hits"] > st["num_hsps"] >= 1
    body = out[1:]
    keys = [(int(r["query_start"]), -int(r["len"]), int(r["ref_start"])) for r in body]
    assert keys == sorted(keys) and len(set(keys)) == len(keys)
    assert (40, 40, 119, 120 // 4 * 382) in [tuple(int(x) for x in r) for r in body]
    assert int(out[0]["len"]) == len(body) and int(out[0]["score"]) == st["num_hits"]
