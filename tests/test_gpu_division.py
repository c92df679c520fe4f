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


@pytest.mark.parametrize("seed", [3, 2027])
def test_branch_free_reciprocal_and_quotient_on_the_gpu(seed):
    """The persistent sweeps' branch-free forms (mfg_selftest_division_fast):
    2^30 pairs per seed, divisors across [2^-130, 2^130] with every eighth
    significand all ones, every eighth + 1 all ones but the last bit, every
    eighth + 2 a power of two.  Where the fast path is taken, the reciprocal
    and the quotient carry the division's bits; the divisors it leaves to the
    division are the all-ones significands and those outside its window."""
    lib = _lib.load()
    counts = (ct.c_int64 * 3)(-1, -1, -1)
    n = 1 << 30
    _lib.check("mfg_selftest_division_fast", lib.mfg_selftest_division_fast(n, seed, counts))
    assert counts[0] == 0, f"{counts[0]} reciprocals differ from 1 / b"
    assert counts[1] == 0, f"{counts[1]} quotients differ from a / b"
    # the all-ones eighth, plus the exponents beyond 2^+-119 (20 of 261)
    assert n // 8 <= counts[2] < n // 8 + n * 24 // 261
