"""Batched outputs copied back to the host in parts (SA_OUT_PARTS_MIN=1 forces
the part-wise copy on a small batch, in a child process, since the library
reads the variable once): every unit's HSP list must equal the one-copy result
of this process, headers included."""
import os
import subprocess
import sys

import numpy as np
import pytest

from segalign_b200 import SeedFilter, build_sub_mat, synth
from tests.helpers import small_workload

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from segalign_b200 import SeedFilter, build_sub_mat, synth
from tests.helpers import small_workload
w = small_workload()
sf = SeedFilter()
sf.initialize_interface(1)
sf.generate_shape_pos("12of19")
sf.initialize_processor(False, 250_000, 19, build_sub_mat(910), 910, 3000, False)
sf.send_ref_write_request(w.target)
sf.generate_seed_pos_table(None, 1, 19, 12)
sf.send_query_write_request(w.query, 0)
L = len(w.query) - 19
units = []
for (a, b) in synth.loguniform_chunks(211, L, 2_000, 250_000).tolist():
    units += [(0, 0, a, b), (0, 1, L - b, L - a)]
units.append((0, 0, 5, 5))
outs = sf.seed_and_filter_batch(units)
np.save(sys.argv[2], np.concatenate([o.view(np.uint32).ravel() for o in outs]))
np.save(sys.argv[3], np.array([len(o) for o in outs], dtype=np.int64))
sf.shutdown_processor()
"""


def _run_here():
    w = small_workload()
    sf = SeedFilter()
    sf.initialize_interface(1)
    sf.generate_shape_pos("12of19")
    sf.initialize_processor(False, 250_000, 19, build_sub_mat(910), 910, 3000, False)
    sf.send_ref_write_request(w.target)
    sf.generate_seed_pos_table(None, 1, 19, 12)
    sf.send_query_write_request(w.query, 0)
    L = len(w.query) - 19
    units = []
    for (a, b) in synth.loguniform_chunks(211, L, 2_000, 250_000).tolist():
        units += [(0, 0, a, b), (0, 1, L - b, L - a)]
    units.append((0, 0, 5, 5))
    outs = sf.seed_and_filter_batch(units)
    return outs


def test_output_in_parts_equals_one_copy(built, tmp_path):
    env = dict(os.environ, SA_OUT_PARTS_MIN="1")
    recs, lens = tmp_path / "recs.npy", tmp_path / "lens.npy"
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT, str(recs), str(lens)], env=env, cwd=ROOT,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    outs = _run_here()
    got_lens = np.load(lens)
    assert list(got_lens) == [len(o) for o in outs]
    assert sum(len(o) - 1 for o in outs) > 100  # enough records for four non-empty parts
    want = np.concatenate([o.view(np.uint32).ravel() for o in outs])
    assert np.array_equal(np.load(recs), want)
