"""Host-side grid preparation, the product's counterpart of the reference's
``PreprocessGrid`` sequence (src/Kernels/load_grid.cpp:405-540).

``prepare`` turns a raw FlowStar mesh into the arrays the iteration path
consumes, calling the C++ restatements in ``libmfgpu.so``:

  SpecifyBC -> ComputeMetrics -> AllocAndInitFlowfield (+ seeded density
  bump) -> SetGhostVariables -> ComputeWeight3D_Node -> FindNodeSYMM

or, with ``device=``, the same chain with ComputeMetrics, CalC2N,
ComputeWeight3D_Node and FindNodeSYMM on a GPU (bit-identical arrays).

The LU-SGS order is the serial build's identity order
(``ReorderCellforLUSGS_0``, grid_polyhedra.cpp:1127-1142).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .meshgen import RawMesh


@dataclass
class PreparedGrid:
    n_node: int
    n_face: int
    n_cell: int
    n_bface: int
    arrays: dict = field(default_factory=dict)  # every mfg_mesh array by name
    q0: np.ndarray = None                       # initial state, SoA [5n]

    @property
    def n(self) -> int:
        return self.n_cell + self.n_bface


def make_params(mach=0.8395, alpha=3.06, beita=0.0, re=1.8140449177e7, T=288.15, gam=1.4,
                gascon=287.053, cfl_start=100.0, cfl_end=None, cfl_nstep=2000, lhs_omga=1.0,
                epsa_r=0.1, ratio_dtmax=1.0e80) -> _lib.Params:
    """Parameter block with the reference's defaults (para_field_global.cpp
    :37-130) and derived values (:150-209)."""
    lib = _lib.load()
    p = _lib.Params()
    lib.mfg_params_default(ct_byref(p))
    p.mach, p.alpha, p.beita, p.re, p.T, p.gam, p.gascon = mach, alpha, beita, re, T, gam, gascon
    p.cfl_start = cfl_start
    p.cfl_end = cfl_start if cfl_end is None else cfl_end
    p.cfl_nstep = int(cfl_nstep)
    p.lhs_omga, p.epsa_r, p.ratio_dtmax = lhs_omga, epsa_r, ratio_dtmax
    _lib.check("mfg_params_derive", lib.mfg_params_derive(ct_byref(p)))
    return p


def ct_byref(obj):
    import ctypes
    return ctypes.byref(obj)


def _raw(mesh: RawMesh, f2c: np.ndarray) -> _lib.RawGrid:
    g = _lib.RawGrid()
    g.n_node, g.n_face, g.n_cell, g.n_bface = mesh.n_node, mesh.n_face, mesh.n_cell, mesh.n_bface
    g.x, g.y, g.z = _lib.ptr(mesh.x), _lib.ptr(mesh.y), _lib.ptr(mesh.z)
    g.nnpf = _lib.ptr(mesh.nnpf, _lib.i32p)
    g.f2n = _lib.ptr(mesh.f2n, _lib.i32p)
    g.f2c = _lib.ptr(f2c, _lib.i32p)
    return g


def prepare(mesh: RawMesh, params: _lib.Params, bump_amp: float = 0.05, bump_sigma: float = 0.1,
            bump_center=(0.5, 0.5, 0.5), device: int | None = None,
            stats: dict | None = None) -> PreparedGrid:
    """Run the preprocessing chain on ``mesh`` (not modified).

    With ``device`` (a CUDA device index) the metrics and node weights are
    computed on that GPU (``mfg_prep_gpu_*``, the same bits as the host
    entries); the initial flow field is set on the host either way.
    ``stats``, if given, receives the seconds of each step ("gpu_kernels_s":
    device time of the GPU kernels alone)."""
    if device is not None:
        return _prepare_gpu(mesh, params, bump_amp, bump_sigma, bump_center, int(device), stats)
    lib = _lib.load()
    mesh_x = np.ascontiguousarray(mesh.x, np.float64)
    mesh = RawMesh(x=mesh_x, y=np.ascontiguousarray(mesh.y, np.float64),
                   z=np.ascontiguousarray(mesh.z, np.float64),
                   nnpf=np.ascontiguousarray(mesh.nnpf, np.int32),
                   f2n=np.ascontiguousarray(mesh.f2n, np.int32), f2c=mesh.f2c,
                   n_cell=mesh.n_cell, n_bface=mesh.n_bface, patches=mesh.patches)
    f2c = np.array(mesh.f2c, dtype=np.int32, copy=True)
    g = _raw(mesh, f2c)
    C, G, F, N = mesh.n_cell, mesh.n_bface, mesh.n_face, mesh.n_node
    n = C + G
    types = np.array([t for _, t in mesh.patches], dtype=np.int32)
    bctype = np.zeros(max(G, 1), dtype=np.int32)
    _lib.check("mfg_prep_specify_bc",
               lib.mfg_prep_specify_bc(ct_byref(g), len(types), _lib.ptr(types, _lib.i32p),
                                       _lib.ptr(bctype, _lib.i32p)))
    A = {name: np.zeros(F) for name in ("xfn", "yfn", "zfn", "area", "xfc", "yfc", "zfc")}
    A.update({name: np.zeros(n) for name in ("xcc", "ycc", "zcc", "vol")})
    _lib.check("mfg_prep_metrics", lib.mfg_prep_metrics(
        ct_byref(g), *[_lib.ptr(A[k]) for k in ("xfn", "yfn", "zfn", "area", "xfc", "yfc", "zfc",
                                                 "xcc", "ycc", "zcc", "vol")]))
    q0 = np.zeros(5 * n)
    bx, by, bz = bump_center
    _lib.check("mfg_prep_init_flow", lib.mfg_prep_init_flow(
        ct_byref(g), ct_byref(params), _lib.ptr(bctype, _lib.i32p),
        *[_lib.ptr(A[k]) for k in ("xfn", "yfn", "zfn", "xcc", "ycc", "zcc")],
        float(bump_amp), float(bump_sigma), float(bx), float(by), float(bz), _lib.ptr(q0)))
    import ctypes
    nc2n = ctypes.c_int64(0)
    _lib.check("mfg_prep_c2n_size", lib.mfg_prep_c2n_size(ct_byref(g), ctypes.byref(nc2n)))
    nb_nodes = int(mesh.nnpf[:G].sum())
    W = dict(wnode=np.zeros(N), nmark=np.zeros(N, np.int32), wbface=np.zeros(max(nb_nodes, 1)),
             nnpc=np.zeros(C, np.int32), c2n=np.zeros(nc2n.value, np.int32),
             wc2n=np.zeros(nc2n.value), nodesymm=np.zeros(N, np.int32),
             xfn_n_symm=np.zeros(N), yfn_n_symm=np.zeros(N), zfn_n_symm=np.zeros(N))
    _lib.check("mfg_prep_node_weights", lib.mfg_prep_node_weights(
        ct_byref(g), _lib.ptr(bctype, _lib.i32p),
        *[_lib.ptr(A[k]) for k in ("xfn", "yfn", "zfn", "xfc", "yfc", "zfc", "xcc", "ycc",
                                    "zcc")],
        _lib.ptr(W["wnode"]), _lib.ptr(W["nmark"], _lib.i32p), _lib.ptr(W["wbface"]),
        _lib.ptr(W["nnpc"], _lib.i32p), _lib.ptr(W["c2n"], _lib.i32p), _lib.ptr(W["wc2n"]),
        _lib.ptr(W["nodesymm"], _lib.i32p), _lib.ptr(W["xfn_n_symm"]),
        _lib.ptr(W["yfn_n_symm"]), _lib.ptr(W["zfn_n_symm"])))
    arrays = dict(f2c=f2c, nnpf=mesh.nnpf, f2n=mesh.f2n, bctype=bctype[:G] if G else bctype)
    arrays.update(A)
    arrays.update(W)
    return PreparedGrid(n_node=N, n_face=F, n_cell=C, n_bface=G, arrays=arrays, q0=q0)


def _contiguous(mesh: RawMesh) -> RawMesh:
    return RawMesh(x=np.ascontiguousarray(mesh.x, np.float64),
                   y=np.ascontiguousarray(mesh.y, np.float64),
                   z=np.ascontiguousarray(mesh.z, np.float64),
                   nnpf=np.ascontiguousarray(mesh.nnpf, np.int32),
                   f2n=np.ascontiguousarray(mesh.f2n, np.int32), f2c=mesh.f2c,
                   n_cell=mesh.n_cell, n_bface=mesh.n_bface, patches=mesh.patches)


def _prepare_gpu(mesh, params, bump_amp, bump_sigma, bump_center, device, stats):
    import time
    lib = _lib.load()
    st = stats if stats is not None else {}
    mesh = _contiguous(mesh)
    f2c = np.array(mesh.f2c, dtype=np.int32, copy=True)
    g = _raw(mesh, f2c)
    C, G, F, N = mesh.n_cell, mesh.n_bface, mesh.n_face, mesh.n_node
    n = C + G
    t0 = time.perf_counter()
    types = np.array([t for _, t in mesh.patches], dtype=np.int32)
    bctype = np.zeros(max(G, 1), dtype=np.int32)
    _lib.check("mfg_prep_specify_bc",
               lib.mfg_prep_specify_bc(ct_byref(g), len(types), _lib.ptr(types, _lib.i32p),
                                       _lib.ptr(bctype, _lib.i32p)))
    t1 = time.perf_counter()
    h = ctypes.c_void_p()
    _lib.check("mfg_prep_gpu_run",
               lib.mfg_prep_gpu_run(ct_byref(g), _lib.ptr(bctype, _lib.i32p), device,
                                    ctypes.byref(h)))
    try:
        t2 = time.perf_counter()
        kms = ctypes.c_double(0.0)
        lib.mfg_prep_gpu_kernel_ms(h, ctypes.byref(kms))
        nc2n = ctypes.c_int64(0)
        _lib.check("mfg_prep_gpu_c2n_size", lib.mfg_prep_gpu_c2n_size(h, ctypes.byref(nc2n)))
        A = {name: np.empty(F) for name in ("xfn", "yfn", "zfn", "area", "xfc", "yfc", "zfc")}
        A.update({name: np.empty(n) for name in ("xcc", "ycc", "zcc", "vol")})
        _lib.check("mfg_prep_gpu_metrics", lib.mfg_prep_gpu_metrics(
            h, *[_lib.ptr(A[k]) for k in ("xfn", "yfn", "zfn", "area", "xfc", "yfc", "zfc",
                                          "xcc", "ycc", "zcc", "vol")]))
        nb_nodes = int(mesh.nnpf[:G].sum())
        W = dict(wnode=np.empty(N), nmark=np.empty(N, np.int32),
                 wbface=np.zeros(max(nb_nodes, 1)), nnpc=np.empty(C, np.int32),
                 c2n=np.empty(nc2n.value, np.int32), wc2n=np.empty(nc2n.value),
                 nodesymm=np.empty(N, np.int32), xfn_n_symm=np.empty(N),
                 yfn_n_symm=np.empty(N), zfn_n_symm=np.empty(N))
        _lib.check("mfg_prep_gpu_node_weights", lib.mfg_prep_gpu_node_weights(
            h, _lib.ptr(W["wnode"]), _lib.ptr(W["nmark"], _lib.i32p), _lib.ptr(W["wbface"]),
            _lib.ptr(W["nnpc"], _lib.i32p), _lib.ptr(W["c2n"], _lib.i32p), _lib.ptr(W["wc2n"]),
            _lib.ptr(W["nodesymm"], _lib.i32p), _lib.ptr(W["xfn_n_symm"]),
            _lib.ptr(W["yfn_n_symm"]), _lib.ptr(W["zfn_n_symm"])))
        t3 = time.perf_counter()
    finally:
        lib.mfg_prep_gpu_destroy(h)
    q0 = np.zeros(5 * n)
    bx, by, bz = bump_center
    _lib.check("mfg_prep_init_flow", lib.mfg_prep_init_flow(
        ct_byref(g), ct_byref(params), _lib.ptr(bctype, _lib.i32p),
        *[_lib.ptr(A[k]) for k in ("xfn", "yfn", "zfn", "xcc", "ycc", "zcc")],
        float(bump_amp), float(bump_sigma), float(bx), float(by), float(bz), _lib.ptr(q0)))
    t4 = time.perf_counter()
    st.update(specify_bc_s=t1 - t0, gpu_run_s=t2 - t1, gpu_kernels_s=kms.value / 1e3,
              gpu_download_s=t3 - t2, init_flow_s=t4 - t3, total_s=t4 - t0)
    arrays = dict(f2c=f2c, nnpf=mesh.nnpf, f2n=mesh.f2n, bctype=bctype[:G] if G else bctype)
    arrays.update(A)
    arrays.update(W)
    return PreparedGrid(n_node=N, n_face=F, n_cell=C, n_bface=G, arrays=arrays, q0=q0)


class DevicePrep:
    """The preprocessing kept in device memory (``mfg_prep_gpu_run``): the
    input of ``Solver.from_device_prep``, which builds the context on the
    device without copying the grid through the host."""

    def __init__(self, mesh: RawMesh, device: int = 0):
        lib = _lib.load()
        self.mesh = _contiguous(mesh)
        self.f2c = np.array(mesh.f2c, dtype=np.int32, copy=True)
        g = _raw(self.mesh, self.f2c)
        self.n_node, self.n_face = self.mesh.n_node, self.mesh.n_face
        self.n_cell, self.n_bface = self.mesh.n_cell, self.mesh.n_bface
        types = np.array([t for _, t in mesh.patches], dtype=np.int32)
        self.bctype = np.zeros(max(self.n_bface, 1), dtype=np.int32)
        _lib.check("mfg_prep_specify_bc",
                   lib.mfg_prep_specify_bc(ct_byref(g), len(types), _lib.ptr(types, _lib.i32p),
                                           _lib.ptr(self.bctype, _lib.i32p)))
        self.handle = ctypes.c_void_p()
        _lib.check("mfg_prep_gpu_run",
                   lib.mfg_prep_gpu_run(ct_byref(g), _lib.ptr(self.bctype, _lib.i32p),
                                        int(device), ctypes.byref(self.handle)))
        self.device = int(device)

    @property
    def n(self) -> int:
        return self.n_cell + self.n_bface

    def init_flow(self, params: _lib.Params, bump_amp: float = 0.05, bump_sigma: float = 0.1,
                  bump_center=(0.5, 0.5, 0.5)) -> np.ndarray:
        """The initial state (AllocAndInitFlowfield + bump + SetGhostVariables),
        computed on the host from the device's centroids and normals."""
        q0 = np.zeros(5 * self.n)
        bx, by, bz = bump_center
        _lib.check("mfg_prep_gpu_init_flow", _lib.load().mfg_prep_gpu_init_flow(
            self.handle, ct_byref(params), float(bump_amp), float(bump_sigma), float(bx),
            float(by), float(bz), _lib.ptr(q0)))
        return q0

    def close(self):
        if self.handle:
            _lib.load().mfg_prep_gpu_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def from_arrays(dims, arrays: dict, q0: np.ndarray) -> PreparedGrid:
    """Wrap arrays already produced elsewhere (e.g. by the reference's own
    preprocessing, as a drop-in caller would pass them)."""
    n_node, n_face, n_cell, n_bface = (int(v) for v in dims)
    return PreparedGrid(n_node=n_node, n_face=n_face, n_cell=n_cell, n_bface=n_bface,
                        arrays=dict(arrays), q0=np.ascontiguousarray(q0, np.float64))


def mesh_struct(pg: PreparedGrid, lusgs_order=None, lusgs_layer=None):
    """Build the ``mfg_mesh`` struct; returns (struct, keepalive list)."""
    keep = []

    def arr(name, dt):
        a = np.ascontiguousarray(pg.arrays[name], dtype=dt)
        keep.append(a)
        return a

    m = _lib.Mesh()
    m.n_node, m.n_face, m.n_cell, m.n_bface = pg.n_node, pg.n_face, pg.n_cell, pg.n_bface
    for k in _lib.MESH_I32 + ("nmark", "nnpc", "c2n", "nodesymm"):
        setattr(m, k, _lib.ptr(arr(k, np.int32), _lib.i32p))
    for k in _lib.MESH_F64_FACE + _lib.MESH_F64_CELL + ("wnode", "wbface", "wc2n", "xfn_n_symm",
                                                         "yfn_n_symm", "zfn_n_symm"):
        setattr(m, k, _lib.ptr(arr(k, np.float64)))
    if lusgs_order is not None:
        a = np.ascontiguousarray(lusgs_order, np.int32)
        keep.append(a)
        m.lusgs_order = _lib.ptr(a, _lib.i32p)
    if lusgs_layer is not None:
        a = np.ascontiguousarray(lusgs_layer, np.int32)
        keep.append(a)
        m.lusgs_layer = _lib.ptr(a, _lib.i32p)
    return m, keep
