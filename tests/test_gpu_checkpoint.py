"""Checkpoint and resume on the GPU: a run stopped after some iterations,
saved, and continued in a new context from the file gives the bits of the
uninterrupted run (FP64 and mixed, with a CFL ramp so that the iteration
count matters)."""
import numpy as np
import pytest

from helpers import assert_bitwise
from minifs_b200 import grid as gr, meshgen
from minifs_b200.solver import Solver

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_resume_is_bit_identical(tmp_path, precision):
    m = meshgen.cube_mesh(10, jitter=0.15, seed=4)
    p = gr.make_params(mach=0.6, alpha=3.0, cfl_start=5.0, cfl_end=20.0, cfl_nstep=8)
    pg = gr.prepare(m, p, bump_amp=0.05, bump_sigma=0.15)
    straight = Solver(pg, p, precision=precision)
    n_all = straight.iterate(10)
    first = Solver(pg, p, precision=precision)
    first.iterate(4)
    first.save_checkpoint(tmp_path / "run.ckpt")
    first.close()
    resumed = Solver(pg, p, precision=precision)
    resumed.load_checkpoint(tmp_path / "run.ckpt")
    assert resumed.iter_done == 4
    n_rest = resumed.iterate(6)
    for f in ("q", "res", "dq", "dqdx"):
        assert_bitwise(resumed.download(f), straight.download(f), f"{precision} {f}")
    assert_bitwise(n_rest.reshape(-1), n_all[4:].reshape(-1), f"{precision} norms")
    assert resumed.dt_extrema == straight.dt_extrema
