"""TEST INFRASTRUCTURE ONLY: ctypes front end of the C oracle
(oracle/minifs_oracle.c, built into oracle/_build/liboracle.so).

``OracleSolver`` takes the preprocessed grid arrays (the same names the
reference harness dumps: f2c, xfn, ..., wc2n) and the derived solver
parameters, and runs the restated iteration path on the CPU.
"""
from __future__ import annotations

import ctypes as ct
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

_i32p = ct.POINTER(ct.c_int32)
_f64p = ct.POINTER(ct.c_double)


class _Grid(ct.Structure):
    _fields_ = [("n_node", ct.c_int32), ("n_face", ct.c_int32), ("n_cell", ct.c_int32),
                ("n_bface", ct.c_int32), ("f2c", _i32p), ("nnpf", _i32p), ("f2n", _i32p),
                ("bctype", _i32p)] + \
               [(k, _f64p) for k in ("xfn", "yfn", "zfn", "area", "xfc", "yfc", "zfc", "xcc",
                                     "ycc", "zcc", "vol", "wnode")] + \
               [("nmark", _i32p), ("wbface", _f64p), ("nnpc", _i32p), ("c2n", _i32p),
                ("wc2n", _f64p), ("nodesymm", _i32p), ("xfn_n_symm", _f64p),
                ("yfn_n_symm", _f64p), ("zfn_n_symm", _f64p)]


class _Params(ct.Structure):
    _fields_ = [(k, ct.c_double) for k in ("gam", "gamm1", "p_bar", "alf_l", "lhs_omga", "rho_s",
                                           "rho_min", "rho_max", "p_min", "p_max", "p_break",
                                           "cfl_start", "cfl_end", "cfl_ratio",
                                           "ratio_dtmax")] + [("cfl_nstep", ct.c_int32)]


class _State(ct.Structure):
    _fields_ = [(k, _f64p) for k in ("q", "res", "dt", "dq", "diag", "dqdx", "dqdy", "dqdz")] + \
               [("dt_max", ct.c_double), ("dt_min", ct.c_double), ("cfl_min", ct.c_double),
                ("iter_done", ct.c_int32)]


_lib = None


def load():
    """Load liboracle.so, compiling it with the system C compiler if needed."""
    global _lib
    if _lib is not None:
        return _lib
    src = os.path.join(HERE, "minifs_oracle.c")
    if (not os.path.exists(LIB_PATH)) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    lib = ct.CDLL(LIB_PATH)
    gp, pp, sp = ct.POINTER(_Grid), ct.POINTER(_Params), ct.POINTER(_State)
    for name in ("mfo_inviscid_flux", "mfo_compute_timestep", "mfo_forward_lusgs",
                 "mfo_calculate_gradient"):
        getattr(lib, name).argtypes = [gp, pp, sp]
        getattr(lib, name).restype = None
    lib.mfo_zero_residuals.argtypes = [gp, sp]
    lib.mfo_residual_norm.argtypes = [gp, sp, _f64p]
    lib.mfo_iterate.argtypes = [gp, pp, sp, ct.c_int32, _f64p]
    lib.mfo_flux_lusgs.argtypes = [_f64p, _f64p, _f64p, _f64p, ct.c_double, ct.c_double,
                                   ct.c_double]
    lib.mfo_roe_flux.argtypes = [_f64p, _f64p, _f64p] + [ct.c_double] * 8
    lib.mfo_update_flow.argtypes = [ct.POINTER(_Params), ct.c_int32, ct.c_int64, _f64p, _f64p]
    lib.mfo_update_flow.restype = None
    _lib = lib
    return lib


def _p(a, t):
    return a.ctypes.data_as(t)


class OracleSolver:
    """CPU oracle bound to one grid.  ``grid`` maps the preprocessing array
    names to numpy arrays; ``params`` maps derived parameter names to values."""

    GRID_I32 = ("f2c", "nnpf", "f2n", "bctype", "nmark", "nnpc", "c2n", "nodesymm")
    GRID_F64 = ("xfn", "yfn", "zfn", "area", "xfc", "yfc", "zfc", "xcc", "ycc", "zcc", "vol",
                "wnode", "wbface", "wc2n", "xfn_n_symm", "yfn_n_symm", "zfn_n_symm")

    def __init__(self, grid: dict, params: dict, q0: np.ndarray, dims):
        self.lib = load()
        n_node, n_face, n_cell, n_bface = (int(v) for v in dims)
        self.keep = {}
        for k in self.GRID_I32:
            self.keep[k] = np.ascontiguousarray(grid[k], dtype=np.int32)
        for k in self.GRID_F64:
            self.keep[k] = np.ascontiguousarray(grid[k], dtype=np.float64)
        g = _Grid()
        g.n_node, g.n_face, g.n_cell, g.n_bface = n_node, n_face, n_cell, n_bface
        for k in self.GRID_I32:
            setattr(g, k, _p(self.keep[k], _i32p))
        for k in self.GRID_F64:
            setattr(g, k, _p(self.keep[k], _f64p))
        self.g = g
        pr = _Params()
        for name, _ in _Params._fields_:
            setattr(pr, name, params[name])
        self.p = pr
        n = n_cell + n_bface
        self.n, self.n_cell = n, n_cell
        self.q = np.ascontiguousarray(q0, dtype=np.float64).copy()
        self.res = np.zeros(5 * n_cell)
        self.dt = np.zeros(n_cell)
        self.dq = np.zeros(5 * n)
        self.diag = np.zeros(n_cell)
        self.dqdx = np.zeros(5 * n)
        self.dqdy = np.zeros(5 * n)
        self.dqdz = np.zeros(5 * n)
        s = _State()
        for k in ("q", "res", "dt", "dq", "diag", "dqdx", "dqdy", "dqdz"):
            setattr(s, k, _p(getattr(self, k), _f64p))
        s.dt_max, s.dt_min, s.cfl_min, s.iter_done = 0.0, 1e40, 0.5 * params["cfl_start"], 0
        self.s = s

    def _call(self, name):
        getattr(self.lib, name)(ct.byref(self.g), ct.byref(self.p), ct.byref(self.s))

    def zero_residuals(self):
        self.lib.mfo_zero_residuals(ct.byref(self.g), ct.byref(self.s))

    def inviscid_flux(self):
        self._call("mfo_inviscid_flux")

    def compute_timestep(self):
        self._call("mfo_compute_timestep")

    def forward_lusgs(self):
        self._call("mfo_forward_lusgs")

    def calculate_gradient(self):
        self._call("mfo_calculate_gradient")

    def step(self):
        self.zero_residuals()
        self.inviscid_flux()
        self.compute_timestep()
        self.forward_lusgs()
        self.calculate_gradient()
        self.s.iter_done += 1

    def iterate(self, n: int) -> np.ndarray:
        norms = np.zeros(5 * n)
        self.lib.mfo_iterate(ct.byref(self.g), ct.byref(self.p), ct.byref(self.s), n,
                             _p(norms, _f64p))
        return norms.reshape(n, 5)

    def residual_norm(self) -> np.ndarray:
        out = np.zeros(5)
        self.lib.mfo_residual_norm(ct.byref(self.g), ct.byref(self.s), _p(out, _f64p))
        return out

    @property
    def dt_extrema(self):
        return self.s.dt_max, self.s.dt_min


def roe_flux(ql, qr, n, area, gam, gamm1, p_bar, alf_l):
    lib = load()
    out = np.zeros(5)
    ql = np.ascontiguousarray(ql, np.float64)
    qr = np.ascontiguousarray(qr, np.float64)
    lib.mfo_roe_flux(_p(out, _f64p), _p(ql, _f64p), _p(qr, _f64p), n[0], n[1], n[2], area, gam,
                     gamm1, p_bar, alf_l)
    return out


def flux_lusgs(q, dq, n, gam, p_bar, lhs_omga):
    lib = load()
    out = np.zeros(5)
    q = np.ascontiguousarray(q, np.float64)
    dq = np.ascontiguousarray(dq, np.float64)
    nn = np.ascontiguousarray(n, np.float64)
    lib.mfo_flux_lusgs(_p(out, _f64p), _p(q, _f64p), _p(dq, _f64p), _p(nn, _f64p), gam, p_bar,
                       lhs_omga)
    return out


def update_flow(q, dq, params):
    """UpdateFlowField3D_CFL3d on every cell of q [5][C] (primitive, no
    ghosts) with dq [5][C]; ``params`` maps gam, p_bar, rho_min, rho_max,
    p_min, p_max to values.  Returns the updated copy of q."""
    lib = load()
    pr = _Params()
    for k, v in params.items():
        setattr(pr, k, v)
    out = np.array(q, np.float64, order="C", copy=True)
    dq = np.ascontiguousarray(dq, np.float64)
    C = out.shape[1]
    lib.mfo_update_flow(ct.byref(pr), C, C, _p(out, _f64p), _p(dq, _f64p))
    return out
