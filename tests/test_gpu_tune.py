"""GPU test of the autotuner: it times candidate tunings of the batched path,
keeps only settings that reproduce the HSP lists exactly, applies the fastest,
and a second call with the same cache applies the stored setting untimed."""
import pytest

from segalign_b200 import SeedFilter, build_sub_mat
from tests.helpers import compare_segments, small_workload

pytestmark = pytest.mark.gpu

@pytest.fixture(scope="module")
def sf(built):
    w = small_workload()
    s = SeedFilter()
    s.initialize_interface(1)
    s.generate_shape_pos("12of19")
    s.initialize_processor(False, 250_000, 19, build_sub_mat(910), 910, 3000, False)
    s.send_ref_write_request(w.target)
    s.generate_seed_pos_table(None, 1, 19, 12)
    s.send_query_write_request(w.query, 0)
    saved = s.get_tuning()
    yield s
    s.set_tuning(**saved)


def test_autotune_keeps_results_and_caches(sf, tmp_path):
    DEFAULT = sf.get_tuning()
    L = 1_000_000 - 19
    units = [(0, r, a, min(a + 125_000, L)) for r in (0, 1) for a in range(0, L, 125_000)]
    want = sf.seed_and_filter_batch(units)
    cache = str(tmp_path / "tune.jsonl")
    res = sf.autotune(units, cache_path=cache, quick=True, repeats=1)
    assert res["candidates"] > 0 and res["rejected"] == 0 and res["from_cache"] == 0
    assert res["ms_best"] <= res["ms_start"]
    tuned = sf.get_tuning()
    knobs = [k for k in DEFAULT if k in res]  # the batched path's knobs (not call_range_ctas)
    assert len(knobs) == 7
    for k in knobs:
        assert tuned[k] == res[k], k
    assert tuned["call_range_ctas"] == DEFAULT["call_range_ctas"]
    for u, (g, x) in enumerate(zip(sf.seed_and_filter_batch(units), want)):
        compare_segments(g, x, f"unit {u} after tuning")
    sf.set_tuning(**DEFAULT)
    again = sf.autotune(units, cache_path=cache, quick=True, repeats=1)
    assert again["from_cache"] == 1 and again["candidates"] == 0
    assert {k: again[k] for k in knobs} == {k: res[k] for k in knobs}
    assert open(cache).read().count("\n") == 1
