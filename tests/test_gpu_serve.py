"""GPU tests of the serving form (sa_serve_*): a request's HSP lists must be
the same whether it runs alone or batched with other requests arriving
concurrently, and equal to the plain path (the C++ seeder calling
sa_seed_and_filter per chunk) on that query alone, bit for bit.  Admission by
device memory must queue requests rather than fail them, and a request that
can never fit must fail with SA_ERR_CAPACITY."""
import threading
import time

import numpy as np
import pytest

import oracle
from segalign_b200 import SeedFilter, SegAlignError, build_sub_mat, host_revcomp
from tests.helpers import compare_segments, random_text, small_workload

pytestmark = pytest.mark.gpu

# small intervals and chunks, so that 1 Mbp requests cross interval borders
IV, OV, CH = 300_000, 50_000, 100_000


@pytest.fixture(scope="module")
def setup(built):
    w = small_workload()
    p = oracle.params()
    idx, pos = oracle.build_table(w.target, p)
    sf = SeedFilter()
    sf.initialize_interface(1)
    sf.generate_shape_pos("12of19")
    sf.initialize_processor(False, 250_000, 19, build_sub_mat(910), 910, 3000, False)
    sf.send_ref_write_request(w.target)
    sf.generate_seed_pos_table(None, 1, 19, 12)
    rng = np.random.default_rng(7)
    q = w.query
    reqs = [q[0:1_000_000], q[123_457:143_457], q[400_000:733_333], q[994_000:999_000], q[10:28],
            q[700_001:850_001], random_text(rng, 250_000, lower=0.02, nfrac=0.001),
            host_revcomp(q[200_000:460_000])]
    want = []
    for t in reqs:
        if len(t) <= 19:
            want.append((np.zeros(0, dtype=np.uint32), np.zeros(0, dtype=np.uint32)))
            continue
        sf.send_query_write_request(t, 1)
        fw, rc, _ = sf.seeder_run(t, buffer=1, strand=3, num_threads=4, interval_size=IV, chunk_size=CH,
                                  interval_overlap=OV)
        want.append((fw, rc))
    return dict(w=w, p=p, idx=idx, pos=pos, sf=sf, reqs=reqs, want=want)


def _check(got, want, what):
    compare_segments(got[0], want[0], what + " plus")
    compare_segments(got[1], want[1], what + " minus")


def test_plain_path_matches_oracle_on_requests(setup):
    """Pins the expected lists: the plain GPU path equals the CPU oracle's
    seeder pipeline for two of the requests."""
    for k in (1, 5):
        fw, rc, _ = oracle.pipeline(setup["p"], setup["w"].target, setup["reqs"][k], setup["idx"], setup["pos"],
                                    strand=3, interval_size=IV, chunk_size=CH, interval_overlap=OV)
        _check(setup["want"][k], (fw, rc), f"request {k}")


def test_each_request_alone(setup):
    sf = setup["sf"]
    sf.serve_start(interval_size=IV, interval_overlap=OV, chunk_size=CH, strands=3)
    try:
        for k, t in enumerate(setup["reqs"]):
            rid = sf.serve_submit(t)
            fw, rc, st = sf.serve_wait(rid, timeout_ms=60_000)
            _check((fw, rc), setup["want"][k], f"request {k} alone")
            assert st["num_hsps"] == len(fw) + len(rc)
            assert st["done_s"] >= st["admit_s"] >= st["submit_s"]
            if len(t) > 19:
                assert st["num_passes"] >= 1 and st["device_bytes"] > 0
    finally:
        sf.serve_stop()


def test_requests_in_a_mix(setup):
    """Requests arrive from four threads while others are on the GPU; passes
    of 2^18 seed slots hold units of several requests."""
    sf = setup["sf"]
    reqs, want = setup["reqs"], setup["want"]
    sf.serve_start(interval_size=IV, interval_overlap=OV, chunk_size=CH, strands=3, pass_slots=1 << 18)
    got, stats, errors = {}, {}, []

    def client(ks, delay):
        try:
            ids = []
            for k in ks:
                ids.append((k, sf.serve_submit(reqs[k])))
                time.sleep(delay)
            for k, rid in ids:
                fw, rc, st = sf.serve_wait(rid, timeout_ms=120_000)
                got[k], stats[k] = (fw, rc), st
        except Exception as e:  # reported below
            errors.append(e)

    try:
        order = [[0, 4], [1, 5, 7], [2, 6], [3]]
        th = [threading.Thread(target=client, args=(ks, 0.002 * (i + 1))) for i, ks in enumerate(order)]
        for t in th:
            t.start()
        for t in th:
            t.join()
    finally:
        sf.serve_stop()
    assert not errors, errors
    for k in range(len(reqs)):
        _check(got[k], want[k], f"request {k} in the mix")
    # the big request took several passes, and some request was admitted
    # while another was still running
    assert stats[0]["num_passes"] > 1
    spans = sorted((s["admit_s"], s["done_s"]) for s in stats.values() if s["num_units"])
    assert any(b[0] < a[1] for a, b in zip(spans, spans[1:]))


def test_admission_by_device_memory(setup):
    """With a budget of about two large requests, the rest wait for memory and
    still complete; a request larger than the whole budget fails."""
    import torch
    sf = setup["sf"]
    reqs, want = setup["reqs"], setup["want"]
    free, _ = torch.cuda.mem_get_info()
    need = 12 * 1_000_000 + (8 << 20)  # about one 1 Mbp request's buffers
    sf.serve_start(interval_size=IV, interval_overlap=OV, chunk_size=CH, strands=3, pass_slots=1 << 20,
                   hbm_reserve=free - 2 * need)
    try:
        ids = [(k, sf.serve_submit(t)) for k, t in enumerate(reqs)]
        big = sf.serve_submit(random_text(np.random.default_rng(9), 4_000_000))
        stats = {}
        for k, rid in ids:
            fw, rc, st = sf.serve_wait(rid, timeout_ms=120_000)
            _check((fw, rc), want[k], f"request {k} under a small budget")
            stats[k] = st
        with pytest.raises(SegAlignError) as ei:
            sf.serve_wait(big, timeout_ms=60_000)
        assert ei.value.code == -8  # SA_ERR_CAPACITY
    finally:
        sf.serve_stop()
    # never more device bytes resident than the budget allows
    events = sorted([(s["admit_s"], s["device_bytes"]) for s in stats.values()] +
                    [(s["done_s"], -s["device_bytes"]) for s in stats.values()], key=lambda e: (e[0], e[1]))
    held = peak = 0
    for _, b in events:
        held += b
        peak = max(peak, held)
    assert peak <= 2 * need + (64 << 20)
