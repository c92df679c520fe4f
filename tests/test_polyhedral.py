"""Mixed hexahedron / triangular-prism meshes (quadrilateral and triangular
faces, cells of 5 and 6 faces, 6 and 8 nodes) and hex blocks with merged
hex pairs (cells of 10 faces and 12 nodes): the host preprocessing and the
C oracle against the reference compiled from its own sources, run on the
same grid file.  Host only."""
import numpy as np
import pytest

from helpers import assert_bitwise, oracle_from
from minifs_b200 import flowstar, grid as gr, meshgen
from oracle import refrun

PREP = ["f2c", "bctype", "xfn", "yfn", "zfn", "area", "xfc", "yfc", "zfc", "xcc", "ycc", "zcc",
        "vol", "wnode", "nmark", "wbface", "nodesymm", "xfn_n_symm", "yfn_n_symm", "zfn_n_symm"]

pytestmark = pytest.mark.skipif(not refrun.available(),
                                reason="reference binaries not built (make -C oracle ref)")


def case(nx=6, ny=5, nz=4, bc=(6, 6, 4, 6, 3, 6), iters=5, jitter=0.15):
    m = meshgen.hexprism_mesh(nx, ny, nz, jitter=jitter, seed=3, bc_types=bc)
    flow = dict(mach=0.5, alpha=3.0, cfl_start=10.0, cfl_end=10.0, n_steps=iters,
                bump_amp=0.05, bump_sigma=0.15, bump_x0=0.5, bump_y0=0.5, bump_z0=0.5)
    p = gr.make_params(mach=0.5, alpha=3.0, cfl_start=10.0, cfl_end=10.0)
    return m, flow, p


def test_mesh_shape():
    m, _, _ = case()
    assert sorted(set(m.nnpf.tolist())) == [3, 4]
    faces_per_cell = np.bincount(m.f2c[0::2], minlength=m.n_cell) + \
        np.bincount(m.f2c[1::2][m.n_bface:], minlength=m.n_cell)
    assert sorted(set(faces_per_cell.tolist())) == [5, 6]


@pytest.mark.parametrize("bc", [(6, 6, 4, 6, 3, 6), (3, 3, 4, 4, 3, 61)])
def test_host_preprocessing_matches_reference(bc, tmp_path):
    m, flow, p = case(bc=bc)
    ref = refrun.run(m, flow, dump_iters="-1", workdir=str(tmp_path))
    pg = gr.prepare(m, p, bump_amp=0.05, bump_sigma=0.15)
    for k in PREP:
        assert_bitwise(pg.arrays[k], ref[k], k)
    assert_bitwise(pg.q0, ref["init.q"], "initial state")

    def cmap(nnpc, c2n, w):
        cells = np.repeat(np.arange(len(nnpc)), nnpc)
        return dict(zip(zip(cells.tolist(), c2n.tolist()), w.tolist()))

    assert cmap(pg.arrays["nnpc"], pg.arrays["c2n"], pg.arrays["wc2n"]) == \
        cmap(ref["nnpc"], ref["c2n"], ref["wc2n"])


def test_oracle_matches_reference(tmp_path):
    m, flow, p = case()
    ref = refrun.run(m, flow, dump_iters="-1", workdir=str(tmp_path))
    pg = gr.prepare(m, p, bump_amp=0.05, bump_sigma=0.15)
    o = oracle_from(pg.arrays, p.as_dict() | {"cfl_nstep": p.cfl_nstep}, pg.q0,
                    (pg.n_node, pg.n_face, pg.n_cell, pg.n_bface))
    for _ in range(flow["n_steps"]):
        o.step()
    assert_bitwise(o.q, ref["final.q"], "oracle state")


def test_grid_file_round_trip(tmp_path):
    m, _, _ = case()
    flowstar.write_grid(m, tmp_path / "g.mfl")
    got, _ = flowstar.read_grid(tmp_path / "g.mfl")
    for k in ("nnpf", "f2n", "f2c"):
        assert np.array_equal(getattr(got, k), getattr(m, k)), k
    assert got.n_bface == m.n_bface


@pytest.mark.parametrize("at_boundary", [False, True])
def test_merged_cells_match_reference(at_boundary, tmp_path):
    m = meshgen.merged_hex_mesh(8, 5, 5, jitter=0.15, seed=3, bc_types=(6, 6, 4, 6, 3, 6),
                                at_boundary=at_boundary)
    _, flow, p = case()
    ref = refrun.run(m, flow, dump_iters="-1", workdir=str(tmp_path))
    pg = gr.prepare(m, p, bump_amp=0.05, bump_sigma=0.15)
    for k in PREP:
        assert_bitwise(pg.arrays[k], ref[k], k)
    assert_bitwise(pg.q0, ref["init.q"], "initial state")
    assert pg.arrays["nnpc"].max() == 12
    o = oracle_from(pg.arrays, p.as_dict() | {"cfl_nstep": p.cfl_nstep}, pg.q0,
                    (pg.n_node, pg.n_face, pg.n_cell, pg.n_bface))
    for _ in range(flow["n_steps"]):
        o.step()
    assert_bitwise(o.q, ref["final.q"], "oracle state")
