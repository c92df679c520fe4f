"""The host-buffer entry point (mfg_iterate_host): the state in, n fused
iterations, state and residual out on a second stream while the last
iteration finishes.  Bit for bit what upload + mfg_iterate + download
give."""
import numpy as np
import pytest

from helpers import assert_bitwise
from minifs_b200 import grid as gr, meshgen
from minifs_b200.solver import Solver

pytestmark = pytest.mark.gpu


def _case():
    m = meshgen.box_mesh(12, 10, 8, jitter=0.15, seed=5, bc_types=(6, 6, 4, 6, 3, 6))
    m.patches = [(i + 1, t) for i, t in enumerate((6, 6, 4, 6, 3, 6))]
    p = gr.make_params(mach=0.6, alpha=2.0, cfl_start=10.0, cfl_end=50.0, cfl_nstep=20)
    return gr.prepare(m, p), p


@pytest.mark.parametrize("n_iter", [1, 3])
@pytest.mark.parametrize("live", [False, True])
def test_iterate_host_equals_upload_iterate_download(n_iter, live):
    pg, p = _case()
    n, C = pg.n, pg.n_cell
    a = Solver(pg, p)
    b = Solver(pg, p)
    a.set_live_bc(live)
    b.set_live_bc(live)
    # a state that is not the prepared one, and the same running dt extrema
    a.iterate(2)
    b.iterate(2)
    q_in = a.download("q")
    q_out = np.full(5 * n, np.nan)
    r_out = np.full(5 * C, np.nan)
    a.iterate_host(n_iter, q_in, q_out, r_out)
    b.upload_q(q_in)
    b.iterate(n_iter)
    assert_bitwise(q_out, b.download("q"), "state")
    assert_bitwise(r_out, b.download("res"), "residual")
    # and the context itself carries on from the same state
    assert_bitwise(a.download("q"), b.download("q"), "context state")
    a.iterate(1)
    b.iterate(1)
    assert_bitwise(a.download("q"), b.download("q"), "next iteration")
    a.close()
    b.close()


def test_iterate_host_one_output_and_norms():
    pg, p = _case()
    n, C = pg.n, pg.n_cell
    a = Solver(pg, p)
    b = Solver(pg, p)
    q_in = pg.q0.copy()
    r_only = np.full(5 * C, np.nan)
    a.iterate_host(2, q_in, None, r_only)
    q_only = np.full(5 * n, np.nan)
    a.iterate_host(2, None, q_only, None)
    b.upload_q(q_in)
    nb = b.iterate(2)
    assert_bitwise(r_only, b.download("res"), "residual alone")
    b.iterate(2)
    assert_bitwise(q_only, b.download("q"), "state alone")
    assert np.all(np.isfinite(nb))
