"""A context built on the device from the device-resident preprocessing
(mfg_create_from_prep) against one built by mfg_create from the host arrays
of the same preprocessing: the same initial state, level sets and sweep grid,
and bit-identical iterations (fused and per routine, FP64 and mixed)."""
import numpy as np
import pytest

from helpers import GOLDEN_CASES, assert_bitwise, load_golden, make_product_params, \
    raw_mesh_from_golden
from minifs_b200 import grid as gr, meshgen
from minifs_b200.solver import Solver

pytestmark = pytest.mark.gpu

INFO = ("n_cell", "n_face", "n_node", "n_bface", "fw_levels", "bw_levels", "max_level_cells",
        "sweep_mode", "sweep_chunks", "sweep_lanes", "sweep_records")


def _both(mesh, params, precision="fp64", **kw):
    host = Solver(gr.prepare(mesh, params, **kw), params, precision=precision)
    prep = gr.DevicePrep(mesh, device=0)
    q0 = prep.init_flow(params, **kw)
    dev = Solver.from_device_prep(prep, params, q0, precision=precision)
    prep.close()  # the context does not depend on it
    return host, dev, q0


def _compare(a, b, what, iters=4, steps=2):
    ia, ib = a.info(), b.info()
    for k in INFO:
        assert ia[k] == ib[k], (what, k, ia[k], ib[k])
    assert_bitwise(b.download("q"), a.download("q"), f"{what} initial state")
    for _ in range(steps):
        a.step()
        b.step()
    assert_bitwise(b.download("q"), a.download("q"), f"{what} per routine")
    a.iterate(iters)
    b.iterate(iters)
    for f in ("q", "res", "dqdx", "dqdy", "dqdz", "dq"):
        assert_bitwise(b.download(f), a.download(f), f"{what} {f}")


@pytest.mark.parametrize("name", GOLDEN_CASES + ("tdtree8",))
def test_device_context_matches_host_context(name):
    d = load_golden(name)
    flow = d["meta"]["case"]["flow"]
    p = make_product_params(d)
    kw = dict(bump_amp=flow["bump_amp"], bump_sigma=flow["bump_sigma"],
              bump_center=(flow["bump_x0"], flow["bump_y0"], flow["bump_z0"]))
    host, dev, q0 = _both(raw_mesh_from_golden(d), p, **kw)
    assert_bitwise(q0, d["init.q"], f"{name} initial state against the reference")
    _compare(host, dev, name)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_device_context_every_boundary_type(precision):
    bc = (3, 6, 4, 61, 5, 10)
    m = meshgen.box_mesh(14, 11, 9, jitter=0.2, seed=3, bc_types=bc, bump=(0.08, 0.2, 0.5))
    m.patches = [(i + 1, t) for i, t in enumerate(bc)]
    p = gr.make_params(mach=0.6, alpha=4.0, cfl_start=10.0)
    host, dev, _ = _both(m, p, precision, bump_amp=0.05, bump_sigma=0.2)
    _compare(host, dev, f"box {precision}")


def test_device_context_bench_grid_and_live_bc():
    m = meshgen.cube_mesh(24, jitter=0.15, seed=1)
    p = gr.make_params(mach=0.5, alpha=2.0, cfl_start=10.0)
    host, dev, _ = _both(m, p)
    host.set_live_bc(True)
    dev.set_live_bc(True)
    _compare(host, dev, "cube24 live", iters=6)
