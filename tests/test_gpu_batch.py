"""Batched cases (mfg_create_batch): independent grids in one context must
each compute exactly what they compute alone -- same bits in every field,
their own CFL ramps and dt extrema -- and the reference's golden states."""
import numpy as np
import pytest

from helpers import assert_bitwise, load_golden, prepare_product

pytestmark = pytest.mark.gpu

FIELDS = ("q", "res", "dt", "diag", "dq", "dqdx", "dqdy", "dqdz")


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _cases():
    """Golden grids plus box grids of other sizes and flow conditions."""
    from minifs_b200 import grid as gr, meshgen
    out = []
    for name in ("cube4", "channel", "ramp5", "tdtree8"):
        d = load_golden(name)
        pg, p = prepare_product(d)
        out.append((name, pg, p, d))
    # the first case limits dt to 3x the smallest (LimitTimeStep's clamp path)
    specs = [((6, 5, 4), 0.5, 0.3, 0.6, 4.0, 12.0, 5, 11, 3.0),
             ((12, 11, 10), 0.65, -2.0, 0.0, 10.0, 10.0, 2000, 3, 1.0e80),
             ((3, 3, 3), 0.3, 4.5, -1.0, 1.0, 6.0, 3, 21, 1.0e80)]
    for (nx, ny, nz), mach, alpha, beita, c0, c1, nstep, seed, ratio in specs:
        m = meshgen.box_mesh(nx, ny, nz, jitter=0.12, seed=seed)
        p = gr.make_params(mach=mach, alpha=alpha, beita=beita, cfl_start=c0, cfl_end=c1,
                           cfl_nstep=nstep, ratio_dtmax=ratio)
        pg = gr.prepare(m, p, bump_amp=0.04, bump_sigma=0.12)
        out.append((f"box{nx}x{ny}x{nz}", pg, p, None))
    return out


def test_batch_equals_single_runs_bitwise():
    from minifs_b200.solver import BatchSolver, Solver
    cases = _cases()
    b = BatchSolver([c[1] for c in cases], [c[2] for c in cases])
    assert b.info()["ncase"] == len(cases)
    iters = 12
    b.calculate_gradient()
    bn = b.iterate(iters)
    got = {f: b.download_cases(f) for f in FIELDS}
    ext = b.dt_extrema
    bnorm = b.residual_norm()
    for k, (name, pg, p, d) in enumerate(cases):
        s = Solver(pg, p)
        s.calculate_gradient()
        sn = s.iterate(iters)
        for f in FIELDS:
            assert_bitwise(got[f][k], s.download(f), f"{name} {f}")
        assert ext[k] == s.dt_extrema, name
        # per-case norms reduce in another order than the single-grid ones
        np.testing.assert_allclose(bn[:, k, :], sn, rtol=1e-13, atol=0)
        np.testing.assert_allclose(bnorm[k], s.residual_norm(), rtol=1e-13, atol=0)
        if d is not None and d["meta"]["case"]["iters"] == iters:
            assert_bitwise(got["q"][k], d["final.q"], f"{name} batched vs reference")
        s.close()
    b.close()


def test_batch_per_routine_equals_fused_and_sweep_modes():
    from minifs_b200.solver import BatchSolver
    cases = _cases()
    grids, params = [c[1] for c in cases], [c[2] for c in cases]
    a, r, m0 = (BatchSolver(grids, params) for _ in range(3))
    m0.set_sweep_mode(0)
    for s in (a, r, m0):
        s.calculate_gradient()
    a.iterate(5)
    m0.iterate(5)
    for _ in range(5):
        r.step()
    for f in FIELDS:
        ref = a.download(f)
        assert_bitwise(r.download(f), ref, f"per-routine vs fused {f}")
        assert_bitwise(m0.download(f), ref, f"per-level vs persistent {f}")
    assert a.dt_extrema == r.dt_extrema == m0.dt_extrema
    for s in (a, r, m0):
        s.close()


def test_batch_upload_round_trip_and_limits():
    from minifs_b200 import _lib
    from minifs_b200.solver import BatchSolver
    cases = _cases()[:3]
    b = BatchSolver([c[1] for c in cases], [c[2] for c in cases])
    qs = b.download_cases("q")
    qs2 = [q * (1.0 + 0.001 * (k + 1)) for k, q in enumerate(qs)]
    b.upload_cases(qs2)
    for k, q in enumerate(b.download_cases("q")):
        assert_bitwise(q, qs2[k], f"case {k} upload")
    with pytest.raises(_lib.MfgError):
        b._call("mfg_set_params", b.params_list[0])
    b.close()


def test_sweep_lanes_identical_and_autotune_restores_state():
    """A wide-level grid (24 cases of 24^3 x 6 cells: ~20k cells per LU-SGS
    level, mixed form).  The autotuner times the lane counts usable with the
    context's chunk grid and leaves the state and dt extrema as they were;
    where W/2 lanes are usable they sweep to the same bits as W lanes, where
    they are not, selecting them is refused."""
    from minifs_b200 import _lib
    from minifs_b200 import grid as gr, meshgen
    from minifs_b200.solver import BatchSolver
    grids, params = [], []
    for k in range(24):
        m = meshgen.cube_mesh(24, jitter=0.1, seed=100 + k)
        p = gr.make_params(mach=0.4 + 0.01 * k, alpha=1.0, cfl_start=10.0)
        grids.append(gr.prepare(m, p, bump_amp=0.05, bump_sigma=0.1))
        params.append(p)
    a = BatchSolver(grids, params, precision="mixed")
    info = a.info()
    w = info["sweep_records"]
    assert info["sweep_lanes"] == w, info
    a.calculate_gradient()
    a.iterate(3)
    q0, e0 = a.download("q"), a.dt_extrema
    tuned = a.autotune_sweeps(2)
    assert set(tuned["ms_per_iter"]) == {str(w), str(w // 2)}
    assert tuned["ms_per_iter"][str(w)] > 0
    assert_bitwise(a.download("q"), q0, "state after autotune")
    assert a.dt_extrema == e0
    half_ok = tuned["ms_per_iter"][str(w // 2)] > 0
    b = BatchSolver(grids, params, precision="mixed")
    if not half_ok:
        assert tuned["lanes_per_cell"] == w
        with pytest.raises(_lib.MfgError):
            b.set_sweep_lanes(w // 2)
        b.close()
        a.close()
        return
    a.set_sweep_lanes(w)
    b.set_sweep_lanes(w // 2)
    b.calculate_gradient()
    b.iterate(3)
    assert_bitwise(a.download("q"), b.download("q"), "before")
    a.iterate(2)
    b.iterate(2)
    for f in ("q", "dq", "diag", "res"):
        assert_bitwise(a.download(f), b.download(f), f"lanes {w} vs {w // 2}: {f}")
    a.close()
    b.close()
