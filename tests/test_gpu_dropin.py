"""The C ABI as a drop-in: the reference's own Base and load_grid code and
its driver sequence, with the shim in place of its four kernel files, on
the GPU -- against the reference's CPU build on the same case files, bit for
bit (state, residual, gradients, dt extrema, per-iteration norms)."""
import numpy as np
import pytest

import dropin
from helpers import assert_bitwise
from minifs_b200 import meshgen
from oracle import refrun

pytestmark = pytest.mark.gpu

FLOW = dict(mach=0.5, alpha=2.0, cfl_start=10.0, cfl_end=10.0, n_steps=10, bump_amp=0.05,
            bump_sigma=0.1, bump_x0=0.5, bump_y0=0.5, bump_z0=0.5)


def _meshes():
    cube = meshgen.cube_mesh(8, jitter=0.15, seed=3)
    bc = (6, 6, 4, 6, 3, 6)
    mixed = meshgen.hexprism_mesh(8, 7, 6, jitter=0.15, seed=4, bc_types=bc)
    return {"cube8": cube, "hexprism": mixed}


@pytest.mark.parametrize("name", ["cube8", "hexprism"])
def test_dropin_matches_reference(name):
    assert dropin.available(), "the drop-in binary is not built"
    m = _meshes()[name]
    got = dropin.run(m, FLOW)
    assert got["returncode"] == 0, got["stderr"][-2000:]
    ref = refrun.run(m, FLOW, dump_iters="-1")
    for k in ("final.q", "final.res", "final.dqdx", "final.dqdy", "final.dqdz",
              "final.dt_extrema"):
        assert_bitwise(got[k], ref[k], f"{name} {k}")
    assert_bitwise(got["norms"], ref["norms"], f"{name} norms of every iteration")
