"""The CUDA path on mixed hexahedron / triangular-prism meshes (quadrilateral
faces take the gradient's face -> node route, triangles the slot record's)
and on hex blocks with merged hex pairs (cells with 5-6 sweep records: the
8-record persistent sweeps; with boundary merges up to 10: one launch per
level): bit for bit against the reference run on the same grid, per routine
and fused; the GPU preprocessing and the device-built context against the
host path."""
import numpy as np
import pytest

from helpers import assert_bitwise
from minifs_b200 import _lib, grid as gr, meshgen
from minifs_b200.compare import state_rel_err
from minifs_b200.solver import Solver
from oracle import refrun

pytestmark = pytest.mark.gpu

ITERS = 12


def case(bc=(6, 6, 4, 6, 3, 6), n=(10, 9, 8)):
    m = meshgen.hexprism_mesh(*n, jitter=0.15, seed=5, bc_types=bc)
    flow = dict(mach=0.6, alpha=2.0, cfl_start=10.0, cfl_end=10.0, n_steps=ITERS,
                bump_amp=0.05, bump_sigma=0.15, bump_x0=0.5, bump_y0=0.5, bump_z0=0.5)
    p = gr.make_params(mach=0.6, alpha=2.0, cfl_start=10.0, cfl_end=10.0)
    pg = gr.prepare(m, p, bump_amp=0.05, bump_sigma=0.15)
    return m, flow, p, pg


@pytest.mark.parametrize("bc", [(6, 6, 4, 6, 3, 6), (3, 3, 4, 4, 3, 61)])
def test_iterations_bitexact_with_reference(bc):
    m, flow, p, pg = case(bc)
    ref = refrun.run(m, flow, dump_iters="-1")
    for fused in (False, True):
        s = Solver(pg, p)
        if fused:
            s.iterate(ITERS)
        else:
            for _ in range(ITERS):
                s.step()
        what = "fused" if fused else "per routine"
        assert_bitwise(s.download("q"), ref["final.q"], f"{what} state")
        assert_bitwise(s.download("res"), ref["final.res"], f"{what} residual")
        for k in ("dqdx", "dqdy", "dqdz"):
            assert_bitwise(s.download(k), ref[f"final.{k}"], f"{what} {k}")
        s.close()


def test_gpu_preprocessing_and_device_context():
    m, flow, p, pg = case()
    dev = gr.prepare(m, p, device=0, bump_amp=0.05, bump_sigma=0.15)
    for k in pg.arrays:
        assert_bitwise(np.asarray(dev.arrays[k]), np.asarray(pg.arrays[k]), k)
    prep = gr.DevicePrep(m, device=0)
    q0 = prep.init_flow(p, bump_amp=0.05, bump_sigma=0.15)
    assert_bitwise(q0, pg.q0, "initial state")
    a = Solver(pg, p)
    b = Solver.from_device_prep(prep, p, q0)
    for key in ("fw_levels", "bw_levels", "sweep_chunks", "sweep_records"):
        assert a.info()[key] == b.info()[key], key
    a.iterate(ITERS)
    b.iterate(ITERS)
    for f in ("q", "res", "dqdx", "dq"):
        assert_bitwise(b.download(f), a.download(f), f)


def test_mixed_precision_close():
    m, flow, p, pg = case()
    a = Solver(pg, p)
    b = Solver(pg, p, precision="mixed")
    a.iterate(ITERS)
    b.iterate(ITERS)
    assert state_rel_err(b.download("q"), a.download("q"), pg.n, p.p_bar)["max_norm"] < 1e-6


def merged_case(at_boundary):
    m = meshgen.merged_hex_mesh(12, 9, 8, jitter=0.15, seed=5, bc_types=(6, 6, 4, 6, 3, 6),
                                at_boundary=at_boundary)
    _, flow, p, _ = case(n=(2, 2, 2))
    pg = gr.prepare(m, p, bump_amp=0.05, bump_sigma=0.15)
    return m, flow, p, pg


@pytest.mark.parametrize("at_boundary", [False, True])
def test_merged_cells_bitexact_with_reference(at_boundary):
    m, flow, p, pg = merged_case(at_boundary)
    ref = refrun.run(m, flow, dump_iters="-1")
    for fused in (False, True):
        s = Solver(pg, p)
        info = s.info()
        if at_boundary:
            assert info["sweep_mode"] == 0 and info["sweep_records"] == 0
        else:
            assert info["sweep_mode"] == 1 and info["sweep_records"] == 8
        if fused:
            s.iterate(ITERS)
        else:
            for _ in range(ITERS):
                s.step()
        what = "fused" if fused else "per routine"
        assert_bitwise(s.download("q"), ref["final.q"], f"{what} state")
        assert_bitwise(s.download("dqdx"), ref["final.dqdx"], f"{what} dqdx")
        s.close()


def test_merged_cells_lanes_mixed_and_device_context():
    m, flow, p, pg = merged_case(False)
    a = Solver(pg, p)
    tuned = a.autotune_sweeps(2)
    assert tuned["lanes_per_cell"] in (4, 8)
    a.iterate(ITERS)
    prep = gr.DevicePrep(m, device=0)
    b = Solver.from_device_prep(prep, p, prep.init_flow(p, bump_amp=0.05, bump_sigma=0.15))
    b.iterate(ITERS)
    assert_bitwise(b.download("q"), a.download("q"), "device-built context")
    c = Solver(pg, p, precision="mixed")
    c.iterate(ITERS)
    assert state_rel_err(c.download("q"), a.download("q"), pg.n, p.p_bar)["max_norm"] < 1e-6


def test_mixed_form_on_cells_beyond_eight_records():
    """Merged cells on the boundary have 10 sweep records: the mixed form
    runs its sweeps one launch per level there.  Those per-level sweeps give
    the persistent mixed sweeps' bits where both run (8-record cells), and
    on the 10-record grid the mixed state stays within 1e-6 of FP64's."""
    m, flow, p, pg = merged_case(False)
    a = Solver(pg, p, precision="mixed")
    b = Solver(pg, p, precision="mixed")
    b.set_sweep_mode(0)
    assert a.info()["sweep_mode"] == 1 and b.info()["sweep_mode"] == 0
    for fused in (True, False):
        if fused:
            a.iterate(ITERS)
            b.iterate(ITERS)
        else:
            a.step()
            b.step()
        for f in ("q", "res", "dqdx", "dq"):
            assert_bitwise(b.download(f), a.download(f), f"mixed per level ({f})")
    a.close()
    b.close()
    m2, _, _, pg2 = merged_case(True)
    f64 = Solver(pg2, p)
    mx = Solver(pg2, p, precision="mixed")
    assert mx.info()["sweep_mode"] == 0 and mx.info()["sweep_records"] == 0
    f64.iterate(ITERS)
    mx.iterate(ITERS)
    err = state_rel_err(mx.download("q"), f64.download("q"), pg2.n, p.p_bar)["max_norm"]
    assert 0.0 < err < 1e-6, err
