"""The launch autotuner (mfg_autotune) and the two persistent sweep kernels:
every knob is timed on the context's own grid, the state is restored after
the trials, and whatever it chooses -- sweep kernels, chunk assignment, sweep
mode, register caps, block sizes -- iterates to the same bits."""
import numpy as np
import pytest

from helpers import assert_bitwise

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cube24():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from minifs_b200 import grid as gr, meshgen
    mesh = meshgen.cube_mesh(24, jitter=0.15, seed=9)
    p = gr.make_params(mach=0.5, alpha=2.0, cfl_start=10.0)
    return p, gr.prepare(mesh, p, bump_amp=0.05, bump_sigma=0.1)


def test_autotune_reports_every_knob_restores_state_and_keeps_bits(cube24):
    from minifs_b200.solver import Solver
    p, pg = cube24
    a = Solver(pg, p)
    a.calculate_gradient()
    a.iterate(2)
    q0, e0 = a.download("q"), a.dt_extrema
    tuned = a.autotune(2)
    knobs = tuned["knobs"]
    assert len(knobs) >= 4, knobs
    for name, k in knobs.items():
        times = list(k["trial_ms_per_iter"].values())
        assert any(t > 0 for t in times), (name, k)
        assert str(k["chosen"]) in k["trial_ms_per_iter"], (name, k)
    assert tuned["ms_per_iter_after"] > 0
    assert_bitwise(a.download("q"), q0, "state after the autotuner")
    assert a.dt_extrema == e0
    # the tuned context and an untuned one iterate to the same bits
    b = Solver(pg, p)
    b.calculate_gradient()
    b.iterate(2)
    a.iterate(3)
    b.iterate(3)
    for f in ("q", "res", "dq", "diag", "dqdx"):
        assert_bitwise(a.download(f), b.download(f), f"tuned vs untuned: {f}")
    a.close()
    b.close()


@pytest.mark.parametrize("mixed", [False, True])
def test_wide_and_deep_sweep_kernels_same_bits(cube24, mixed):
    from minifs_b200 import _lib
    from minifs_b200.solver import Solver
    p, pg = cube24
    lib = _lib.load()
    out = {}
    for kind in (0, 1):
        assert lib.mfg_set_sweep_kernel(kind) == 0
        try:
            s = Solver(pg, p, precision="mixed" if mixed else "fp64")
        finally:
            lib.mfg_set_sweep_kernel(-1)
        assert s.info()["sweep_kernel"] == kind
        s.calculate_gradient()
        s.iterate(3)
        out[kind] = {f: s.download(f) for f in ("q", "res", "dq")}
        s.close()
    for f in out[0]:
        assert_bitwise(out[1][f], out[0][f], f"wide vs deep kernels: {f}")


@pytest.mark.parametrize("mixed", [False, True])
def test_lane_per_face_gathers_same_bits(cube24, mixed):
    """The face gather and gradient sums with one lane per face (the sums
    passed from lane to lane in face order) against one thread per cell:
    every field and every iteration's residual norms bit for bit, fused and
    per routine."""
    from minifs_b200 import _lib
    from minifs_b200.solver import Solver
    p, pg = cube24
    prec = "mixed" if mixed else "fp64"
    a, b = Solver(pg, p, precision=prec), Solver(pg, p, precision=prec)
    b.set_gather_lanes(4)
    with pytest.raises(_lib.MfgError):
        b.set_gather_lanes(8)  # tetrahedra: four faces per cell
    for s in (a, b):
        s.calculate_gradient()
    na, nb = a.iterate(4), b.iterate(4)
    assert_bitwise(nb.reshape(-1), na.reshape(-1), f"{prec} norms")
    for s in (a, b):
        s.step()
    for f in ("q", "res", "dt", "diag", "dq", "dqdx", "dqdy", "dqdz"):
        assert_bitwise(b.download(f), a.download(f), f"{prec} lanes per face: {f}")
    assert_bitwise(b.residual_norm(), a.residual_norm(), f"{prec} routine norm")
    a.close()
    b.close()


@pytest.mark.parametrize("mixed", [False, True])
def test_lane_per_face_gathers_hexahedra_and_prisms(mixed):
    """Eight lanes per cell (hexahedra and prisms, 5 and 6 faces, walls,
    symmetry and far field): the same bits as one thread per cell."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from minifs_b200 import _lib, grid as gr, meshgen
    from minifs_b200.solver import Solver
    m = meshgen.hexprism_mesh(10, 9, 8, jitter=0.15, seed=5, bc_types=(6, 6, 4, 6, 3, 6))
    p = gr.make_params(mach=0.6, alpha=2.0, cfl_start=10.0, cfl_end=10.0)
    pg = gr.prepare(m, p, bump_amp=0.05, bump_sigma=0.15)
    prec = "mixed" if mixed else "fp64"
    a, b = Solver(pg, p, precision=prec), Solver(pg, p, precision=prec)
    with pytest.raises(_lib.MfgError):
        b.set_gather_lanes(4)  # cells of six faces
    b.set_gather_lanes(8)
    for s in (a, b):
        s.calculate_gradient()
    na, nb = a.iterate(4), b.iterate(4)
    assert_bitwise(nb.reshape(-1), na.reshape(-1), f"{prec} norms")
    for f in ("q", "res", "dt", "diag", "dq", "dqdx", "dqdy", "dqdz"):
        assert_bitwise(b.download(f), a.download(f), f"{prec} eight lanes: {f}")
    a.close()
    b.close()
