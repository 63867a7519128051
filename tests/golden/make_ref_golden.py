"""Records the reference's own SeedAndFilter outputs as golden fixtures.

The reference's seed-filter translation units (src/seed_filter.cu,
repeat_masker_src/seed_filter.cu, common/seed_filter_interface.cu,
common/seed_pos_table.cu, common/ntcoding.cpp) are compiled unmodified by
`make -C oracle ref_kernels` into oracle/_ref/ and driven by
oracle/ref_harness.cu.  This script runs them on a GPU over the cases of
tests/ref_cases.py and writes tests/golden/ref_calls.npz: per call the
reference's full output (header row first; the header's ref_start/query_start,
which the reference leaves unset, are recorded as 0), plus a digest of each
case's inputs.  Run from the repository root on a machine with a GPU:

    python tests/golden/make_ref_golden.py [output.npz]
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from tests import ref_cases  # noqa: E402


def main():
    out_path = sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "ref_calls.npz")
    arrays, meta = {}, []
    for case in ref_cases.fixture_cases():
        res = ref_cases.reference_run(case)
        for k, (c, r) in enumerate(zip(case["calls"], res)):
            arrays[f"{case['name']}_{k}"] = r["segments"].view(np.uint32).reshape(-1, 4)
        meta.append({"name": case["name"], "digest": case["digest"], "ncalls": len(case["calls"]),
                     "num_hits": [int(r["num_hits"]) for r in res], "num_seeds": [int(r["num_seeds"]) for r in res],
                     "hsps": [int(r["num_hsps"]) for r in res]})
        print(case["name"], "calls", len(res), "hits", sum(m for m in meta[-1]["num_hits"]),
              "hsps", sum(meta[-1]["hsps"]), flush=True)
    arrays["meta_json"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(out_path, **arrays)
    print("wrote", out_path)


if __name__ == "__main__":
    main()
