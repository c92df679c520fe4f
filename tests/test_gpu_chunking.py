"""The persistent LU-SGS sweeps on grids wide and deep enough to reach every
path of their tables -- increments read from the block's shared-memory ring,
from global memory (same chunk, older than the ring) and from other chunks
(polled in L2) -- with each chunk assignment the library offers (the
balanced vote and the transverse monotone grids, MFG_CHUNK_*): the same bits
as the one-launch-per-level sweeps and as the CPU oracle."""
import numpy as np
import pytest

from helpers import assert_bitwise

pytestmark = pytest.mark.gpu

KINDS = {"vote": 0, "transverse_xy": 1, "transverse_xz": 2, "transverse_yz": 3}
# transverse on any axis pair: the chunking the model finds best among them
ANY_TRANSVERSE = 4


@pytest.fixture(scope="module")
def cube32():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from minifs_b200 import grid as gr, meshgen
    mesh = meshgen.cube_mesh(32, jitter=0.15, seed=3)
    p = gr.make_params(mach=0.5, alpha=2.0, cfl_start=10.0)
    pg = gr.prepare(mesh, p, bump_amp=0.05, bump_sigma=0.1)
    return mesh, p, pg


def _run(pg, p, kind, iters, mode=1):
    from minifs_b200 import _lib
    from minifs_b200.solver import Solver
    lib = _lib.load()
    assert lib.mfg_set_chunking(kind) == 0
    try:
        s = Solver(pg, p)
    finally:
        lib.mfg_set_chunking(-1)
    info = s.info()
    if mode == 0:
        s.set_sweep_mode(0)
    s.calculate_gradient()
    norms = s.iterate(iters)
    out = {f: s.download(f) for f in ("q", "res", "dq", "diag", "dt", "dqdx")}
    out["norms"] = norms
    s.close()
    return info, out


def test_every_chunking_same_bits_and_every_table_path(cube32):
    """196,608 cells, 128 levels per sweep: each assignment's tables read
    increments from the ring, from global memory and from other chunks, and
    every assignment (and the per-level launches) gives the same bits."""
    _, p, pg = cube32
    iters = 3
    _, ref = _run(pg, p, -1, iters, mode=0)
    for name, kind in KINDS.items():
        info, out = _run(pg, p, kind, iters)
        assert info["sweep_mode"] == 1 and info["sweep_chunking"] == kind, (name, info)
        for k in range(2):  # forward, backward
            assert info["sweep_ring_records"][k] > 0, (name, k, info)
            assert info["sweep_cross_records"][k] > 0, (name, k, info)
            if name == "vote":
                # the vote assignment mixes the order of the chunk's cells enough
                # that some dependencies are older than the ring
                assert info["sweep_global_records"][k] >= 0
        for f in ("q", "res", "dq", "diag", "dt", "dqdx"):
            assert_bitwise(out[f], ref[f], f"{name}: {f}")
        np.testing.assert_array_equal(out["norms"], ref["norms"], err_msg=name)


def test_wide_levels_reach_the_global_fallback_and_two_passes():
    """A batch of 24 cubes of 24^3 x 6 cells (about 20,000 cells per LU-SGS
    level, 140 per chunk and level): levels take two passes of the block's
    lane groups, the 512-position ring holds only the last few levels, so
    some increments of the block's own chunk are read back from global
    memory; the persistent sweeps still give the per-level sweeps' bits."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from minifs_b200 import grid as gr, meshgen
    from minifs_b200.solver import BatchSolver
    grids, params = [], []
    for k in range(24):
        m = meshgen.cube_mesh(24, jitter=0.1, seed=300 + k)
        p = gr.make_params(mach=0.4 + 0.01 * k, alpha=1.0, cfl_start=10.0)
        grids.append(gr.prepare(m, p, bump_amp=0.05, bump_sigma=0.1))
        params.append(p)
    from minifs_b200 import _lib
    lib = _lib.load()
    out = {}
    for mode in (1, 0):
        lib.mfg_set_sweep_kernel(0)  # one block per SM: wide chunk levels
        try:
            b = BatchSolver(grids, params)
        finally:
            lib.mfg_set_sweep_kernel(-1)
        info = b.info()
        if mode == 1:
            assert info["sweep_mode"] == 1, info
            assert min(info["sweep_global_records"]) > 0, info
            assert min(info["sweep_ring_records"]) > 0, info
            assert min(info["sweep_cross_records"]) > 0, info
            assert info["sweep_model_us"][0] > 0, info
        else:
            b.set_sweep_mode(0)
        b.calculate_gradient()
        b.iterate(2)
        out[mode] = {f: b.download(f) for f in ("q", "res", "dq", "diag")}
        b.close()
    for f in out[1]:
        assert_bitwise(out[1][f], out[0][f], f"persistent vs per-level: {f}")
