"""The benchmark's per-knot FLOP constants equal the operation counts of the
reference's own device functions (oracle/ref_shim/flop_count.cpp), when that
counter has been built from the reference sources."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
COUNTER = os.path.join(ROOT, "oracle", "_ref", "flop_count_iiwa14")


@pytest.mark.skipif(not os.path.exists(COUNTER), reason="reference FLOP counter not built")
def test_bench_knot_flops_match_reference_counts():
    sys.path.insert(0, ROOT)
    import bench
    out = subprocess.run([COUNTER], check=True, capture_output=True, text=True).stdout
    counts = json.loads(out)
    assert counts["nq"] == 7
    for k, v in bench.REF_KNOT_FLOPS.items():
        assert counts[k] == v, (k, counts[k], v)
