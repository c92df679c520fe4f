"""The sweeps' division by a precomputed reciprocal on the GPU
(mfg_selftest_division): 2^30 pseudo-random pairs across the exponent range
give the division's bits."""
import ctypes as ct

import pytest

from minifs_b200 import _lib

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed", [7, 99])
def test_division_by_reciprocal_on_the_gpu(seed):
    lib = _lib.load()
    bad = ct.c_int64(-1)
    _lib.check("mfg_selftest_division", lib.mfg_selftest_division(1 << 30, seed, ct.byref(bad)))
    assert bad.value == 0
