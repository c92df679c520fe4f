"""Mixed-precision form (MFG_PREC_MIXED): FP32 Roe averages / dissipation,
LU-SGS off-diagonal products and gradient; FP64 residual accumulation, Diag
division, norm and update.  Checked against the FP64 form on the same inputs:
its error after a transient, and that it reaches the same residual drop with
a state within 1e-6 (relative) of the FP64 one."""
import numpy as np
import pytest

from helpers import assert_bitwise

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _rel_err(a, b, n):
    """Largest per-component error relative to that component's magnitude."""
    out = []
    for k in range(5):
        x, y = a[k * n:(k + 1) * n], b[k * n:(k + 1) * n]
        out.append(np.max(np.abs(x - y)) / max(np.max(np.abs(y)), 1e-30))
    return max(out)


def _state_err(a, b, n, p_bar):
    """State error on physical scales: density against density, velocity
    against the speed, gauge pressure against the absolute pressure (v and
    the gauge pressure are near zero in these flows: no scale of their own)."""
    from minifs_b200.compare import state_rel_err
    return state_rel_err(a, b, n, p_bar)["max_norm"]


def _pair(pg, p):
    from minifs_b200.solver import Solver
    return Solver(pg, p, precision="fp64"), Solver(pg, p, precision="mixed")


def test_mixed_transient_close_to_fp64():
    from minifs_b200 import grid as gr, meshgen
    m = meshgen.cube_mesh(10, jitter=0.15, seed=2)
    p = gr.make_params(mach=0.8, alpha=1.25, cfl_start=20.0)
    pg = gr.prepare(m, p, bump_amp=0.05, bump_sigma=0.1)
    a, b = _pair(pg, p)
    assert b.info()["precision"] == 1
    for s in (a, b):
        s.calculate_gradient()
    na, nb = a.iterate(30), b.iterate(30)
    # tolerance: FP32 rounding of the dissipation and off-diagonal terms
    assert _state_err(b.download("q"), a.download("q"), pg.n, p.p_bar) < 1e-6
    # norms: the density norm (the one the residual drop is measured on)
    # closely; the others relative to their largest value, loosely (the
    # momentum normal to the flow has residuals near zero)
    np.testing.assert_allclose(nb[:, 0], na[:, 0], rtol=1e-3)
    dev = np.abs(nb - na) / na.max(axis=0)
    assert dev.max() < 5e-2, dev.max(axis=0)
    # the residual (a sum of cancelling fluxes) and the gradient (FP32) of
    # the drifted transient stay within a few percent of their magnitudes
    C = pg.n_cell
    assert _rel_err(b.download("res"), a.download("res"), C) < 5e-2
    assert _rel_err(b.download("dqdx"), a.download("dqdx"), pg.n) < 5e-2
    a.close()
    b.close()


def test_mixed_reaches_same_drop_and_state():
    """Channel with a wall bump, CFL 30: both forms below a 1e-6 residual
    drop, states within 1e-6 relative."""
    from minifs_b200 import grid as gr, meshgen
    m = meshgen.channel_mesh(24, 6, 6, jitter=0.1, seed=5)
    p = gr.make_params(mach=0.7, alpha=0.0, cfl_start=30.0)
    pg = gr.prepare(m, p, bump_amp=0.0, bump_sigma=0.1)
    a, b = _pair(pg, p)
    for s in (a, b):
        s.calculate_gradient()
    na, nb = a.iterate(500), b.iterate(500)
    drop_a = na[-1, 0] / na[0, 0]
    drop_b = nb[-1, 0] / nb[0, 0]
    assert drop_a < 1e-6 and drop_b < 1e-6, (drop_a, drop_b)
    assert _state_err(b.download("q"), a.download("q"), pg.n, p.p_bar) < 1e-6
    a.close()
    b.close()


def test_mixed_batched_and_per_routine():
    """A mixed batch computes each case as a mixed single context does, and
    the per-routine calls match the fused iteration."""
    from minifs_b200 import grid as gr, meshgen
    from minifs_b200.solver import BatchSolver, Solver
    grids, params = [], []
    for n, mach, seed in ((5, 0.5, 1), (7, 0.7, 2)):
        m = meshgen.cube_mesh(n, jitter=0.1, seed=seed)
        p = gr.make_params(mach=mach, alpha=2.0, cfl_start=10.0)
        grids.append(gr.prepare(m, p, bump_amp=0.05, bump_sigma=0.1))
        params.append(p)
    b = BatchSolver(grids, params, precision="mixed")
    b.calculate_gradient()
    b.iterate(6)
    qs = b.download_cases("q")
    for k, (pg, p) in enumerate(zip(grids, params)):
        s = Solver(pg, p, precision="mixed")
        r = Solver(pg, p, precision="mixed")
        s.calculate_gradient()
        r.calculate_gradient()
        s.iterate(6)
        for _ in range(6):
            r.step()
        np.testing.assert_array_equal(qs[k], s.download("q"))
        np.testing.assert_array_equal(r.download("q"), s.download("q"))
        s.close()
        r.close()
    b.close()


def test_mixed_per_level_sweeps_match_persistent():
    """The mixed form's sweeps one launch per level give the persistent mixed
    sweeps' bits (cube with far field and the LimitTimeStep clamp active)."""
    from minifs_b200 import grid as gr, meshgen
    from minifs_b200.solver import Solver
    m = meshgen.cube_mesh(12, jitter=0.15, seed=3)
    p = gr.make_params(mach=0.5, alpha=2.0, cfl_start=10.0)
    pg = gr.prepare(m, p, bump_amp=0.05, bump_sigma=0.1)
    a = Solver(pg, p, precision="mixed")
    b = Solver(pg, p, precision="mixed")
    b.set_sweep_mode(0)
    assert a.info()["sweep_mode"] == 1 and b.info()["sweep_mode"] == 0
    a.iterate(6)
    b.iterate(6)
    for f in ("q", "res", "dq", "dqdx"):
        assert_bitwise(b.download(f), a.download(f), f"mixed per level ({f})")
    a.close()
    b.close()


def test_mixed_form_with_fp64_flux():
    """mfg_set_flux_fp64: the mixed form's face flux from the FP64 kernel
    gives the FP64 form's residual bit for bit on the same state; switching
    back restores the FP32 dissipation; the FP64 form refuses to go FP32."""
    from minifs_b200 import _lib, grid as gr, meshgen
    from minifs_b200.solver import Solver
    m = meshgen.box_mesh(10, 8, 6, jitter=0.15, seed=2, bc_types=(6, 6, 4, 6, 3, 6))
    m.patches = [(i + 1, t) for i, t in enumerate((6, 6, 4, 6, 3, 6))]
    p = gr.make_params(mach=0.7, alpha=1.0, cfl_start=30.0)
    pg = gr.prepare(m, p)
    a = Solver(pg, p)
    b = Solver(pg, p, precision="mixed")
    b.set_flux_fp64(True)
    for s in (a, b):
        s.zero_residuals()
        s.inviscid_flux()
    assert np.array_equal(a.download("res"), b.download("res"))
    b.set_flux_fp64(False)
    b.zero_residuals()
    b.inviscid_flux()
    assert not np.array_equal(a.download("res"), b.download("res"))
    a.set_flux_fp64(True)
    with pytest.raises(_lib.MfgError) as e:
        a.set_flux_fp64(False)
    assert e.value.code == -6
    b.set_flux_fp64(True)
    b.iterate(5)
    assert np.all(np.isfinite(b.download("q")))
