"""The CPU baseline of the batched leg: the reference's threaded build over a
seeded subset of the batch's cases, one after another (no GPU)."""
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
