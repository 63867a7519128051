"""Pins the oracle's seeding half to the reference's own code.

oracle/_ref/libref_ntcoding.so is the reference's common/ntcoding.cpp
compiled from its source tree (oracle/Makefile `ref`).  The oracle's
character coding, shape parsing, k-mer keys and host reverse complement must
agree with it on random texts that include lowercase, N, separators and
other IUPAC letters.  The product's C++ host seeder is checked the same way.
"""
import ctypes as C

import numpy as np
import pytest

import oracle

SHAPES = {"12of19": "TTT0T00TT00T0T0TTTT", "14of22": "TTT0T0TT00TT00T0T0TTTT", "1101011": "TT0T0TT"}
ALPHABET = np.frombuffer(b"ACGTACGTACGTACGTacgtNn&RYK", dtype=np.uint8)


@pytest.fixture(scope="module")
def ref(built):
    L = oracle.ref_ntcoding()
    if L is None:
        pytest.skip("reference ntcoding not built (reference tree absent)")
    return L


def _text(seed, n):
    rng = np.random.default_rng(seed)
    return rng.choice(ALPHABET, size=n).tobytes()


@pytest.mark.parametrize("name", list(SHAPES))
def test_kmer_keys_match_reference(ref, name):
    pat = SHAPES[name]
    k = ref.ref_generate_shape_pos(pat.encode())
    p = oracle.params(shape=name)
    assert k == p.kmer_size
    assert all(ref.ref_is_transition_at_pos(t) == 1 for t in range(k))
    for seed in range(3):
        # mostly-valid texts so that both valid and invalid windows occur
        rng = np.random.default_rng(100 + seed)
        t = bytearray(rng.choice(np.frombuffer(b"ACGT", dtype=np.uint8), size=4000).tobytes())
        noise = _text(seed, 4000)
        for i in rng.choice(4000, size=40, replace=False):
            t[i] = noise[i]
        t = bytes(t)
        buf = C.create_string_buffer(t)
        for pos in range(0, len(t) - len(pat)):
            want = ref.ref_get_kmer_index_at_pos(buf, pos, len(pat))
            got = oracle.lib().or_kmer_index(t, pos, C.byref(p))
            assert got == want, (name, pos)


def test_host_seeder_matches_reference_keys(ref, built):
    from segalign_b200 import host_seeds

    ref.ref_generate_shape_pos(SHAPES["12of19"].encode())
    t = _text(5, 3000).upper().replace(b"R", b"A")
    buf = C.create_string_buffer(t)
    want = []
    for j in range(0, len(t) - 19):
        k = ref.ref_get_kmer_index_at_pos(buf, j, 19)
        if k != (1 << 31):
            want.append((k << 32) + j)
            want.extend(((k ^ (2 << (2 * tt))) << 32) + j for tt in range(12))
    got = host_seeds(t, 0, len(t) - 19, transition=True)
    assert got.tolist() == want


def test_revcomp_matches_reference(ref):
    for seed in range(4):
        t = _text(seed, 5000)
        dst = C.create_string_buffer(len(t))
        src = C.create_string_buffer(t)
        ref.ref_revcomp(dst, src, 0, 0, len(t))
        n_valid = sum(ch in b"ACGTacgtnN&" for ch in t)
        want = dst.raw[:n_valid]
        assert oracle.revcomp_text(t) == want


def test_product_revcomp_matches_oracle(built):
    from segalign_b200 import host_revcomp

    t = _text(9, 20000)
    assert host_revcomp(t) == oracle.revcomp_text(t)
