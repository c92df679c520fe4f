"""The LU-SGS sweeps divide by the diagonal through its reciprocal, formed
before the dividend is known (div_by_recip, Markstein's correction steps).
On the CPU: the same steps with the C library's fma give the division's
bits on pseudo-random pairs across the exponent range."""
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("seed", [1, 2024])
def test_division_by_reciprocal_is_correctly_rounded(tmp_path, seed):
    exe = tmp_path / "div_check"
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-o", str(exe),
                    os.path.join(HERE, "div_by_recip_check.c"), "-lm"], check=True)
    out = subprocess.run([str(exe), "20000000", str(seed)], check=True, capture_output=True,
                         text=True).stdout
    assert int(out.strip()) == 0
