"""The bench's CPU-side legs (no GPU): the batched leg's baseline (the
reference's threaded build over a seeded subset of the batch's cases, one
after another) and the reference arm's JSON line."""
import json

import pytest

from oracle import refrun


@pytest.mark.skipif(not refrun.available(tdtree=True),
                    reason="the reference's TDTree build (oracle/_ref) is not built")
def test_batched_cpu_sample():
    import bench
    bw = bench.batched_workload(64)
    r = bench.cpu_sample_batched(bw, ncase=2, iters=1)
    json.dumps(r)  # goes into the bench line as it is
    assert r["kind"] == "reference" and r["unit"] == bench.UNIT
    assert r["value"] > 0 and r["cores"] >= 1
    assert bw["name"] in r["sample"] and "1 full iterations each" in r["sample"]
    # the same seeded subset every time
    assert r["sample"].split(" (")[0] == \
        bench.cpu_sample_batched(bw, ncase=2, iters=1)["sample"].split(" (")[0]


@pytest.mark.skipif(not refrun.available(tdtree=True),
                    reason="the reference's TDTree build (oracle/_ref) is not built")
def test_reference_arm_line():
    """`bench.py --impl reference`: one JSON line on the FP64 workload from
    the reference's own CPU build, with the keys the line contract names."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1",
                          "--warmup", "0"], cwd=root, capture_output=True, text=True,
                         timeout=600, check=True).stdout
    lines = [json.loads(x) for x in out.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    d = lines[0]
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["config"]["workload"] == "cube64x6_M0.5_a2_cfl10_fp64"
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
