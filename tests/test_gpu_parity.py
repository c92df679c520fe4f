"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle and
the reference's golden outputs.  FP64 form: bit-for-bit, with the stated
floating-point tolerances of the path (1e-12 relative per residual entry,
1e-10 in state after 100 iterations) asserted as well for the record."""
import numpy as np
import pytest

from helpers import (GOLDEN_CASES, assert_bitwise, golden_params, load_golden, oracle_from,
                     prepare_product)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _pair(name):
    """Product solver on the GPU and oracle on the CPU, same inputs."""
    from minifs_b200.solver import Solver
    d = load_golden(name)
    pg, p = prepare_product(d)
    s = Solver(pg, p)
    o = oracle_from(pg.arrays, golden_params(d), pg.q0, (pg.n_node, pg.n_face, pg.n_cell,
                                                          pg.n_bface))
    return d, s, o


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_each_routine_bitexact(name):
    d, s, o = _pair(name)
    s.calculate_gradient()
    o.calculate_gradient()
    assert_bitwise(s.download("dqdx"), o.dqdx, "initial gradient")
    iters = d["meta"]["case"]["iters"]
    for it in range(iters):
        s.zero_residuals()
        o.zero_residuals()
        s.inviscid_flux()
        o.inviscid_flux()
        assert_bitwise(s.download("res"), o.res, f"it{it} InviscidFlux res")
        s.compute_timestep()
        o.compute_timestep()
        assert_bitwise(s.download("dt"), o.dt, f"it{it} ComputeTimeStep dt")
        assert s.dt_extrema == tuple(o.dt_extrema)
        s.forward_lusgs()
        o.forward_lusgs()
        assert_bitwise(s.download("diag"), o.diag, f"it{it} Diag")
        assert_bitwise(s.download("dq"), o.dq, f"it{it} DQ")
        assert_bitwise(s.download("q"), o.q, f"it{it} state")
        s.calculate_gradient()
        o.calculate_gradient()
        for ax in "xyz":
            assert_bitwise(s.download("dqd" + ax), getattr(o, "dqd" + ax), f"it{it} dqd{ax}")
        s.iter_done += 1
        o.s.iter_done += 1
        key = f"it{it}.q"
        if key in d:
            assert_bitwise(s.download("q"), d[key], f"it{it} state vs reference")
    assert_bitwise(s.download("q"), d["final.q"], "final state vs reference")
    s.close()


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_fused_iteration_bitexact(name):
    d, s, o = _pair(name)
    s.calculate_gradient()
    iters = d["meta"]["case"]["iters"]
    norms = s.iterate(iters)
    onorms = o.iterate(iters)
    assert_bitwise(s.download("q"), d["final.q"], "fused state vs reference")
    assert_bitwise(s.download("res"), d["final.res"], "fused res vs reference")
    assert_bitwise(s.download("dqdx"), d["final.dqdx"], "fused gradient vs reference")
    assert_bitwise(s.download("q"), o.q, "fused state vs oracle")
    assert s.dt_extrema == tuple(o.dt_extrema)
    # norms: parallel reduction order, so a tolerance
    np.testing.assert_allclose(norms, onorms, rtol=1e-13, atol=0)
    np.testing.assert_allclose(norms.reshape(-1), d["norms"], rtol=1e-13, atol=0)
    s.close()


def test_fused_equals_per_routine_and_is_deterministic():
    _, a, _ = _pair("ramp5")
    _, b, _ = _pair("ramp5")
    _, c, _ = _pair("ramp5")
    a.iterate(7)
    for _ in range(7):
        b.step()
    c.iterate(3)
    c.iterate(4)
    for f in ("q", "res", "dt", "diag", "dq", "dqdx", "dqdy", "dqdz"):
        assert_bitwise(a.download(f), b.download(f), f"fused vs per-routine {f}")
        assert_bitwise(a.download(f), c.download(f), f"7 vs 3+4 {f}")


def test_tdtree_renumbered_grid():
    """The reference's own TDTree ordering (METIS renumbering): the GPU runs
    the serial arithmetic on it, which is also the TDTree build's state."""
    d, s, o = _pair("tdtree8")
    iters = d["meta"]["case"]["iters"]
    s.calculate_gradient()
    s.iterate(iters)
    assert_bitwise(s.download("q"), d["final.q"], "GPU vs serial reference on renumbered grid")
    assert_bitwise(s.download("q"), d["tdtree.final.q"], "GPU vs TDTree build")
    info = s.info()
    assert info["fw_levels"] > 1 and info["bw_levels"] > 1


def test_config1_cube16_100_iterations():
    """Configuration 1 (16^3 x 6 tets, M 0.5, alpha 2, CFL 10, 100 iterations):
    state after 100 iterations against the oracle."""
    from minifs_b200 import grid as gr, meshgen
    from minifs_b200.solver import Solver
    m = meshgen.cube_mesh(16, jitter=0.15, seed=1)
    p = gr.make_params(mach=0.5, alpha=2.0, cfl_start=10.0)
    pg = gr.prepare(m, p, bump_amp=0.05, bump_sigma=0.1)
    s = Solver(pg, p)
    o = oracle_from(pg.arrays, p.as_dict() | {"cfl_nstep": p.cfl_nstep}, pg.q0,
                    (pg.n_node, pg.n_face, pg.n_cell, pg.n_bface))
    s.calculate_gradient()
    norms = s.iterate(100)
    onorms = o.iterate(100)
    q, oq = s.download("q"), o.q
    n = pg.n
    for k in range(5):
        blk = slice(k * n, (k + 1) * n)
        scale = np.max(np.abs(oq[blk])) or 1.0
        assert np.max(np.abs(q[blk] - oq[blk])) / scale <= 1e-10
    res = s.download("res")
    C = pg.n_cell
    for k in range(5):
        blk = slice(k * C, (k + 1) * C)
        scale = np.max(np.abs(o.res[blk])) or 1.0
        assert np.max(np.abs(res[blk] - o.res[blk])) / scale <= 1e-12
    assert_bitwise(q, oq, "cube16 100-iteration state")
    np.testing.assert_allclose(norms, onorms, rtol=1e-12)
    assert norms[-1, 0] < norms[0, 0]


def test_upload_download_round_trip_and_errors():
    from minifs_b200 import _lib
    d, s, _ = _pair("cube4")
    q = s.download("q")
    q2 = q.copy()
    q2[: s.grid.n_cell] *= 1.01
    s.upload_q(q2)
    assert_bitwise(s.download("q"), q2, "upload/download")
    with pytest.raises(_lib.MfgError):
        s._call("mfg_download", 99, _lib.ptr(q))
    s.zero_residuals()
    assert not s.download("res").any()
    s.close()


@pytest.mark.parametrize("name", ["cube4", "tdtree8"])
def test_sweep_modes_identical(name):
    """Per-level launches and the persistent dataflow sweeps give the same bits."""
    d, a, _ = _pair(name)
    _, b, _ = _pair(name)
    assert a.info()["sweep_mode"] == 1, "persistent sweeps should be the default on B200"
    b.set_sweep_mode(0)
    for s in (a, b):
        s.calculate_gradient()
        s.iterate(4)
        s.step()
    for f in ("q", "dq", "diag", "res", "dqdx"):
        assert_bitwise(a.download(f), b.download(f), f"sweep modes {f}")


def test_bounded_wait_reports_timeout_and_context_survives():
    """Failure detection without a fault: a sweep whose first level is withheld
    must give up waiting, report MFG_ERR_TIMEOUT, and leave a usable context."""
    d, s, o = _pair("ramp5")
    s.calculate_gradient()
    o.calculate_gradient()
    s.iterate(2)
    o.iterate(2)
    before = s.download("dq")
    assert s.selftest_sweep_timeout(2_000_000) == -4
    assert_bitwise(s.download("dq"), before, "state untouched by the self-test")
    s.iterate(3)
    o.iterate(3)
    assert_bitwise(s.download("q"), o.q, "iterations after the self-test")
