"""The drop-in binary (the reference's Base and load_grid code, its driver
sequence and the shim over libmfgpu) is built and links; without a GPU it
stops the way the reference stops on an error: a message and exit(1)."""
import pytest

import dropin
from minifs_b200 import meshgen


@pytest.mark.skipif(not dropin.available(), reason="built only where the reference sources are")
def test_dropin_reports_missing_device_like_the_reference():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present: tests/test_gpu_dropin.py runs it")
    m = meshgen.cube_mesh(2, jitter=0.1)
    r = dropin.run(m, dict(mach=0.5, alpha=2.0, cfl_start=10.0, cfl_end=10.0, n_steps=2))
    assert r["returncode"] == 1
    assert "mfg_create" in r["stderr"] and "no usable CUDA device" in r["stderr"]
