"""Python mirror of the reference's ``src/Kernels`` interface, backed by the
CUDA path in ``libmfgpu.so``.

The reference's free functions take a ``PolyGrid*`` and read globals; here
they take a ``Solver`` that owns the device context and the globals that
the reference keeps at file scope (``iter_done``, ``dt_max``, ``dt_min``):

    ZeroResiduals(s); InviscidFlux(s, None, 0); ComputeTimeStep(s)
    ForwardLUSGS(s, 0); PassInterfaceData(s); CalculateGradient(s)
    s.iter_done += 1

is the body of ``main.cpp:201-291``.  ``Solver.iterate`` runs the same body
with fused kernels captured in a CUDA graph.
"""
from __future__ import annotations

import ctypes as ct

import numpy as np

from . import _lib
from .grid import PreparedGrid, mesh_struct


class Solver:
    def __init__(self, grid: PreparedGrid, params: _lib.Params, device: int = 0,
                 precision: str = "fp64", lusgs_order=None, lusgs_layer=None):
        self.lib = _lib.load()
        self.grid = grid
        self.params = params
        self.iter_done = 0
        m, keep = mesh_struct(grid, lusgs_order, lusgs_layer)
        q0 = np.ascontiguousarray(grid.q0, np.float64)
        self._ctx = ct.c_void_p()
        _lib.check("mfg_create", self.lib.mfg_create(ct.byref(m), ct.byref(params), _lib.ptr(q0),
                                                     int(device), _lib.PREC[precision],
                                                     ct.byref(self._ctx)))
        del keep

    # -- lifetime ----------------------------------------------------------
    def close(self):
        if self._ctx:
            self.lib.mfg_destroy(self._ctx)
            self._ctx = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def ctx(self):
        return self._ctx

    def _call(self, name, *args):
        _lib.check(name, getattr(self.lib, name)(self._ctx, *args))

    # -- the iteration path ------------------------------------------------
    def zero_residuals(self):
        self._call("mfg_zero_residuals")

    def inviscid_flux(self):
        self._call("mfg_inviscid_flux")

    def compute_timestep(self):
        self._call("mfg_compute_timestep", int(self.iter_done))

    def forward_lusgs(self):
        self._call("mfg_forward_lusgs")

    def calculate_gradient(self):
        self._call("mfg_calculate_gradient")

    def step(self):
        """One ``main.cpp:201-291`` iteration through the per-routine calls."""
        self.zero_residuals()
        self.inviscid_flux()
        self.compute_timestep()
        self.forward_lusgs()
        self.calculate_gradient()
        self.iter_done += 1

    def iterate(self, n: int, norms: bool = True) -> np.ndarray | None:
        """``n`` fused iterations (CUDA graph); returns the residual norms
        after each iteration, shape ``[n, 5]``."""
        out = np.zeros(5 * n) if norms else None
        self._call("mfg_iterate", int(n), int(self.iter_done),
                   _lib.ptr(out) if norms else None)
        self.iter_done += n
        return out.reshape(n, 5) if norms else None

    def iterate_host(self, n: int, q_in: np.ndarray, q_out: np.ndarray | None,
                     res_out: np.ndarray | None):
        """End-to-end form: host state in, ``n`` iterations, host state and
        residual out."""
        self._call("mfg_iterate_host", int(n), int(self.iter_done), _lib.ptr(q_in),
                   _lib.ptr(q_out) if q_out is not None else None,
                   _lib.ptr(res_out) if res_out is not None else None, None)
        self.iter_done += n

    def profile_phases(self, n: int) -> dict:
        """``n`` fused iterations with CUDA events between phases; returns
        summed device milliseconds per phase."""
        out = np.zeros(len(_lib.PHASES))
        self._call("mfg_profile_phases", int(n), int(self.iter_done), _lib.ptr(out))
        self.iter_done += n
        return dict(zip(_lib.PHASES, out.tolist()))

    def set_sweep_mode(self, mode: int):
        """0 = one kernel per LU-SGS level, 1 = persistent dataflow sweeps."""
        self._call("mfg_set_sweep_mode", int(mode))

    def selftest_sweep_timeout(self, spin_cycles: int = 2_000_000) -> int:
        """Run the bounded-wait self-test; returns the status code."""
        return int(self.lib.mfg_selftest_sweep_timeout(self._ctx, int(spin_cycles)))

    def set_stream(self, stream_handle: int):
        """Issue the context's work on this cudaStream_t (e.g. torch's)."""
        _lib.check("mfg_set_stream", self.lib.mfg_set_stream(self._ctx, ct.c_void_p(stream_handle)))

    def residual_norm(self) -> np.ndarray:
        out = np.zeros(5)
        self._call("mfg_residual_norm", _lib.ptr(out))
        return out

    @property
    def dt_extrema(self):
        a, b = ct.c_double(), ct.c_double()
        self._call("mfg_get_dt_extrema", ct.byref(a), ct.byref(b))
        return a.value, b.value

    # -- data --------------------------------------------------------------
    def download(self, field: str) -> np.ndarray:
        C, n = self.grid.n_cell, self.grid.n
        size = {"q": 5 * n, "res": 5 * C, "dt": C, "dq": 5 * n, "dqdx": 5 * n, "dqdy": 5 * n,
                "dqdz": 5 * n, "diag": C}[field]
        out = np.empty(size)
        self._call("mfg_download", _lib.FIELD[field], _lib.ptr(out))
        return out

    def upload_q(self, q: np.ndarray):
        q = np.ascontiguousarray(q, np.float64)
        self._call("mfg_upload", _lib.FIELD["q"], _lib.ptr(q))

    def sync(self):
        self._call("mfg_sync")

    def info(self) -> dict:
        inf = _lib.Info()
        self._call("mfg_info_get", ct.byref(inf))
        return {k: getattr(inf, k) for k, _ in inf._fields_}


# Reference-named entry points (src/Kernels/*.h), operating on a Solver.

def ZeroResiduals(s: Solver):  # cal_flux.h:24
    s.zero_residuals()


def InviscidFlux(s: Solver, limit=None, level: int = 0):  # cal_flux.h:27
    if limit is not None or level != 0:
        raise ValueError("the reference calls InviscidFlux(grid, NULL, 0) only (main.cpp:209-227)")
    s.inviscid_flux()


def ComputeTimeStep(s: Solver):  # compute_timestep.h:24
    s.compute_timestep()


def ForwardLUSGS(s: Solver, level: int = 0):  # forward_lusgs.h:23
    if level != 0:
        raise ValueError("only the finest level (0) exists")
    s.forward_lusgs()


def PassInterfaceData(s: Solver):  # load_grid.h:37, a no-op without MPI
    return None


def CalculateGradient(s: Solver):  # cal_gradient.h:23
    s.calculate_gradient()


def AllocAndCalQuantityGradient(s: Solver):  # cal_gradient.h:22
    s.calculate_gradient()
