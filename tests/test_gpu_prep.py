"""Mesh preprocessing on the GPU (mfg_prep_gpu_*): the metrics, cell-node
lists and node weights against the reference's own outputs (golden cases)
and against the host restatement (larger meshes, every boundary type, the
centroid-correction branch), bit for bit; bad meshes give the host's error
code without any out-of-range access."""
import numpy as np
import pytest

from helpers import GOLDEN_CASES, assert_bitwise, load_golden, make_product_params, \
    raw_mesh_from_golden
from minifs_b200 import _lib, grid as gr, meshgen

pytestmark = pytest.mark.gpu

REF_ARRAYS = ["f2c", "bctype", "xfn", "yfn", "zfn", "area", "xfc", "yfc", "zfc", "xcc", "ycc",
              "zcc", "vol", "wnode", "nmark", "wbface", "nodesymm", "xfn_n_symm", "yfn_n_symm",
              "zfn_n_symm"]
ALL_ARRAYS = REF_ARRAYS + ["nnpc", "c2n", "wc2n"]


def _prep_both(mesh, params, **kw):
    host = gr.prepare(mesh, params, **kw)
    stats = {}
    dev = gr.prepare(mesh, params, device=0, stats=stats, **kw)
    return host, dev, stats


def _same(host, dev, what):
    for k in ALL_ARRAYS:
        assert_bitwise(dev.arrays[k], host.arrays[k], f"{what} {k}")
    assert_bitwise(dev.q0, host.q0, f"{what} q0")


@pytest.mark.parametrize("name", GOLDEN_CASES + ("tdtree8",))
def test_gpu_preprocessing_matches_reference(name):
    d = load_golden(name)
    flow = d["meta"]["case"]["flow"]
    params = make_product_params(d)
    kw = dict(bump_amp=flow["bump_amp"], bump_sigma=flow["bump_sigma"],
              bump_center=(flow["bump_x0"], flow["bump_y0"], flow["bump_z0"]))
    host, dev, _ = _prep_both(raw_mesh_from_golden(d), params, **kw)
    for k in REF_ARRAYS:
        assert_bitwise(dev.arrays[k], d[k], f"{name} {k}")
    assert_bitwise(dev.q0, d["init.q"], f"{name} initial state")
    _same(host, dev, name)


@pytest.mark.parametrize("spec", [
    # every boundary type: wall, far field, symmetry, far field (mod), a type
    # outside those (weights in the third pass), interface (no weights)
    dict(n=(18, 14, 11), bc=(3, 6, 4, 61, 5, 10), jitter=0.2, bump=(0.08, 0.2, 0.5)),
    # walls meeting symmetry planes and far field along edges and corners
    # (jitter 0.25 h: close to the largest that keeps every tet positive)
    dict(n=(9, 23, 7), bc=(4, 4, 3, 6, 3, 6), jitter=0.25, bump=None),
    # a slab thinner than the centroid-correction threshold (1e-10): the
    # CorrectCellCentroid moves happen in most cells
    dict(n=(6, 5, 4), bc=(6,) * 6, jitter=0.1, bump=None, lz=2e-10),
])
def test_gpu_preprocessing_matches_host(spec):
    nx, ny, nz = spec["n"]
    m = meshgen.box_mesh(nx, ny, nz, lz=spec.get("lz", 1.0), jitter=spec["jitter"], seed=7,
                         bc_types=spec["bc"], bump=spec["bump"])
    m.patches = [(i + 1, t) for i, t in enumerate(spec["bc"])]
    params = gr.make_params(mach=0.6, alpha=4.0, cfl_start=10.0)
    host, dev, stats = _prep_both(m, params, bump_amp=0.05, bump_sigma=0.2)
    _same(host, dev, str(spec["n"]))
    assert stats["gpu_kernels_s"] > 0.0


def test_gpu_preprocessing_cube_bench_grid():
    """The benchmark's grid family at 24^3 x 6 cells."""
    m = meshgen.cube_mesh(24, jitter=0.15, seed=1)
    params = gr.make_params(mach=0.5, alpha=2.0, cfl_start=10.0)
    host, dev, _ = _prep_both(m, params)
    _same(host, dev, "cube24")


def test_gpu_preprocessing_thin_slab_moves_centroids():
    """The slab case above does reach CorrectCellCentroid's branch."""
    m = meshgen.box_mesh(6, 5, 4, lz=2e-10, jitter=0.1, seed=7, bc_types=(6,) * 6)
    m.patches = [(i + 1, 6) for i in range(6)]
    params = gr.make_params(mach=0.6, alpha=4.0, cfl_start=10.0)
    dev = gr.prepare(m, params, device=0)
    zc = dev.arrays["zcc"][:m.n_cell]
    # each move is about 1e-10 along a face normal, as large as the slab is
    # thick: most centroids end up outside it
    assert np.count_nonzero((zc < 0.0) | (zc > 2e-10)) > m.n_cell // 2


def _raw_for(m, f2c):
    g = _lib.RawGrid()
    g.n_node, g.n_face, g.n_cell, g.n_bface = m.n_node, m.n_face, m.n_cell, m.n_bface
    g.x, g.y, g.z = _lib.ptr(m.x), _lib.ptr(m.y), _lib.ptr(m.z)
    g.nnpf = _lib.ptr(m.nnpf, _lib.i32p)
    g.f2n = _lib.ptr(m.f2n, _lib.i32p)
    g.f2c = _lib.ptr(f2c, _lib.i32p)
    return g


def _gpu_run_code(m, f2c, bctype):
    import ctypes
    lib = _lib.load()
    h = ctypes.c_void_p()
    rc = lib.mfg_prep_gpu_run(ctypes.byref(_raw_for(m, f2c)), _lib.ptr(bctype, _lib.i32p), 0,
                              ctypes.byref(h))
    if rc == 0:
        lib.mfg_prep_gpu_destroy(h)
    else:
        assert not h.value
    return rc


def _specified(m):
    """f2c after SpecifyBC and the boundary types (cube_mesh: all far field)."""
    f2c = np.array(m.f2c, np.int32, copy=True)
    G = m.n_bface
    bctype = np.full(max(G, 1), 6, np.int32)
    f2c[1:2 * G:2] = np.arange(G, dtype=np.int32) + m.n_cell
    return f2c, bctype


@pytest.mark.parametrize("where", ["node", "node_negative", "cell", "cell_interior_c2"])
def test_gpu_preprocessing_rejects_out_of_range_indices(where):
    """Checked on the device before any kernel indexes with them: bad mesh,
    nothing computed."""
    m = meshgen.cube_mesh(3, jitter=0.1)
    m.x = np.ascontiguousarray(m.x)
    m.y = np.ascontiguousarray(m.y)
    m.z = np.ascontiguousarray(m.z)
    m.nnpf = np.ascontiguousarray(m.nnpf, np.int32)
    m.f2n = np.array(m.f2n, np.int32, copy=True)
    f2c, bctype = _specified(m)
    assert _gpu_run_code(m, f2c, bctype) == 0
    if where == "node":
        m.f2n[len(m.f2n) // 2] = m.n_node
    elif where == "node_negative":
        m.f2n[5] = -1
    elif where == "cell":
        f2c[0] = m.n_cell
    else:
        f2c[2 * (m.n_face - 1) + 1] = -3
    assert _gpu_run_code(m, f2c, bctype) == -7


def test_gpu_preprocessing_reports_bad_volume():
    """An inverted cell: MFG_ERR_BADMESH, as the host entry (the reference
    exits, CellVolCentroid)."""
    m = meshgen.cube_mesh(2, jitter=0.0)
    g = m.n_bface
    m.f2n[3 * g + 1], m.f2n[3 * g + 2] = m.f2n[3 * g + 2], m.f2n[3 * g + 1]
    m.x = m.x.copy()
    m.x[13] = 5.0
    p = gr.make_params(mach=0.5, alpha=2.0, cfl_start=10.0)
    for dev in (None, 0):
        with pytest.raises(_lib.MfgError) as e:
            gr.prepare(m, p, device=dev)
        assert e.value.code == -7


def test_gpu_preprocessing_rejects_bad_arguments():
    import ctypes
    lib = _lib.load()
    m = meshgen.cube_mesh(2, jitter=0.0)
    f2c, bctype = _specified(m)
    m.nnpf = np.ascontiguousarray(m.nnpf, np.int32)
    m.f2n = np.ascontiguousarray(m.f2n, np.int32)
    h = ctypes.c_void_p()
    g = _raw_for(m, f2c)
    assert lib.mfg_prep_gpu_run(ctypes.byref(g), _lib.ptr(bctype, _lib.i32p), 0, None) == -1
    assert lib.mfg_prep_gpu_run(ctypes.byref(g), _lib.ptr(bctype, _lib.i32p), 99,
                                ctypes.byref(h)) == -8
    g.n_bface = g.n_face + 1
    assert lib.mfg_prep_gpu_run(ctypes.byref(g), _lib.ptr(bctype, _lib.i32p), 0,
                                ctypes.byref(h)) == -1
    g.n_bface = m.n_bface
    nnpf = m.nnpf.copy()
    nnpf[4] = 0
    g.nnpf = _lib.ptr(nnpf, _lib.i32p)
    assert lib.mfg_prep_gpu_run(ctypes.byref(g), _lib.ptr(bctype, _lib.i32p), 0,
                                ctypes.byref(h)) == -7
