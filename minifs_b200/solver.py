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

    @classmethod
    def from_device_prep(cls, prep, params: _lib.Params, q0: np.ndarray,
                         precision: str = "fp64") -> "Solver":
        """A solver whose context is built on the device from a
        ``grid.DevicePrep`` (``mfg_create_from_prep``; identity LU-SGS
        order), on the preprocessing's device."""
        self = cls.__new__(cls)
        self.lib = _lib.load()
        self.grid = PreparedGrid(n_node=prep.n_node, n_face=prep.n_face, n_cell=prep.n_cell,
                                 n_bface=prep.n_bface, arrays={},
                                 q0=np.ascontiguousarray(q0, np.float64))
        self.params = params
        self.iter_done = 0
        self._ctx = ct.c_void_p()
        _lib.check("mfg_create_from_prep", self.lib.mfg_create_from_prep(
            prep.handle, ct.byref(params), _lib.ptr(self.grid.q0), _lib.PREC[precision],
            ct.byref(self._ctx)))
        return self

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

    def set_ghost_variables(self):
        """``SetGhostVariables``: ghost states from the current inner cells."""
        self._call("mfg_set_ghost_variables")

    def set_live_bc(self, on: bool):
        """Recompute the ghost states every iteration (after the LU-SGS
        update, where ``main.cpp:286`` has the call commented out) instead
        of keeping the initial ones."""
        self._call("mfg_set_live_bc", 1 if on else 0)
        self.live_bc = bool(on)

    def set_order(self, order: int, venkat_k: float = 5.0):
        """The reference's ``order`` switch: 1 first order (default), 2
        second order unlimited, 3 Barth-Jespersen, 4 Venkatakrishnan."""
        self._call("mfg_set_order", int(order), float(venkat_k))

    def set_flux_fp64(self, on: bool):
        """Mixed form: the Roe flux wholly in FP64 (True) or with its
        dissipation in FP32 (False, the default)."""
        self._call("mfg_set_flux_fp64", 1 if on else 0)

    def step(self):
        """One ``main.cpp:201-291`` iteration through the per-routine calls."""
        self.zero_residuals()
        self.inviscid_flux()
        self.compute_timestep()
        self.forward_lusgs()
        if getattr(self, "live_bc", False):
            self.set_ghost_variables()
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

    def iterate_host(self, n: int, q_in: np.ndarray | None, q_out: np.ndarray | None,
                     res_out: np.ndarray | None, norms: np.ndarray | None = None):
        """End-to-end form: host state in (None: keep the context's), ``n``
        iterations, host state and residual out (either may be None);
        ``norms`` (optional, [n][ncase][5]) receives the residual norms of
        every iteration."""
        if norms is not None and norms.size < 5 * n * getattr(self, "ncase", 1):
            raise ValueError("norms needs 5 entries per iteration and case")
        self._call("mfg_iterate_host", int(n), int(self.iter_done),
                   _lib.ptr(q_in) if q_in is not None else None,
                   _lib.ptr(q_out) if q_out is not None else None,
                   _lib.ptr(res_out) if res_out is not None else None,
                   _lib.ptr(norms) if norms is not None else None)
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

    def set_sweep_lanes(self, lanes: int):
        """Persistent sweeps: lanes per cell (the record slots per cell W)."""
        self._call("mfg_set_sweep_lanes", int(lanes))

    def set_gather_lanes(self, lanes: int):
        """Face gather and gradient sums: 0 = one thread per cell, 4 or 8 = one
        lane per face (as the grid's cells allow); identical results."""
        self._call("mfg_set_gather_lanes", int(lanes))

    def autotune_sweeps(self, n_trial: int = 3) -> dict:
        """Time both lane counts on this grid and keep the faster; the state
        is left as it was.  Returns the choice and the ms per iteration."""
        ms = np.zeros(2)
        self._call("mfg_autotune_sweeps", int(n_trial), int(self.iter_done), _lib.ptr(ms))
        info = self.info()
        w = info["sweep_records"]
        return {"lanes_per_cell": info["sweep_lanes"], "chunks": info["sweep_chunks"],
                "ms_per_iter": {str(w): float(ms[0]), str(w // 2): float(ms[1])}}

    def autotune(self, n_trial: int = 3, rebuild: bool = True) -> dict:
        """mfg_autotune: every launch knob timed on this grid (coordinate
        descent), the fastest kept, the state left as it was (rebuild=False:
        the sweep kernels and chunk tables as they are).  Returns, per knob,
        the ms per fused iteration of each candidate and the choice."""
        rep = _lib.TuneReport()
        self._call("mfg_autotune", int(n_trial), int(self.iter_done), 0 if rebuild else 1,
                   ct.byref(rep))
        knobs = {}
        for k in range(rep.n_knobs):
            name = _lib.KNOBS.get(rep.knob[k], str(rep.knob[k]))
            knobs[name] = {"trial_ms_per_iter": {str(rep.cand[k][i]): float(rep.ms[k][i])
                                                 for i in range(rep.n_cand[k])},
                           "chosen": int(rep.chosen[k])}
        return {"knobs": knobs, "ms_per_iter_before": float(rep.ms_initial),
                "ms_per_iter_after": float(rep.ms_final)}

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
                "dqdz": 5 * n, "diag": C, "limiter": 5 * C}[field]
        out = np.empty(size)
        self._call("mfg_download", _lib.FIELD[field], _lib.ptr(out))
        return out

    def save_checkpoint(self, path):
        """The solver state between iterations (state, iteration count, dt
        extrema) to `path` (``mfg_checkpoint_write``)."""
        import os
        q = self.download("q")
        mx, mn = self.dt_extrema
        _lib.check("mfg_checkpoint_write", self.lib.mfg_checkpoint_write(
            os.fsencode(os.fspath(path)), self.grid.n_cell, self.grid.n, int(self.iter_done),
            float(mx), float(mn), _lib.ptr(q)))

    def load_checkpoint(self, path):
        """Restore a state saved by ``save_checkpoint`` on the same grid: the
        run continues with the bits it would have had uninterrupted."""
        import os
        q = np.empty(5 * self.grid.n)
        it = ct.c_int32(0)
        mx, mn = ct.c_double(0.0), ct.c_double(0.0)
        _lib.check("mfg_checkpoint_read", self.lib.mfg_checkpoint_read(
            os.fsencode(os.fspath(path)), self.grid.n_cell, self.grid.n, ct.byref(it),
            ct.byref(mx), ct.byref(mn), _lib.ptr(q)))
        self.upload_q(q)
        self._call("mfg_set_dt_extrema", mx.value, mn.value)
        self.iter_done = int(it.value)

    def upload_q(self, q: np.ndarray):
        q = np.ascontiguousarray(q, np.float64)
        self._call("mfg_upload", _lib.FIELD["q"], _lib.ptr(q))

    def sync(self):
        self._call("mfg_sync")

    def info(self) -> dict:
        inf = _lib.Info()
        self._call("mfg_info_get", ct.byref(inf))
        return {k: (list(getattr(inf, k)) if isinstance(getattr(inf, k), ct.Array)
                    else getattr(inf, k)) for k, _ in inf._fields_}


class BatchSolver(Solver):
    """Independent cases solved together in one context (``mfg_create_batch``):
    one launch per kernel and per LU-SGS level covers every case.  Each case
    gets the bits it would get alone; fields come back per case."""

    def __init__(self, grids, params, device: int = 0, precision: str = "fp64"):
        self.lib = _lib.load()
        self.grids = list(grids)
        self.params_list = list(params)
        if len(self.grids) != len(self.params_list) or not self.grids:
            raise ValueError("one Params per grid, at least one case")
        self.ncase = len(self.grids)
        self.iter_done = 0
        meshes, keeps, q0s = [], [], []
        for g in self.grids:
            m, keep = mesh_struct(g)
            meshes.append(m)
            keeps.append(keep)
            q0s.append(np.ascontiguousarray(g.q0, np.float64))
        marr = (_lib.Mesh * self.ncase)(*meshes)
        parr = (_lib.Params * self.ncase)(*self.params_list)
        qarr = (_lib.f64p * self.ncase)(*[_lib.ptr(q) for q in q0s])
        self._ctx = ct.c_void_p()
        _lib.check("mfg_create_batch",
                   self.lib.mfg_create_batch(self.ncase, marr, parr, qarr, int(device),
                                             _lib.PREC[precision], ct.byref(self._ctx)))
        del keeps
        self.cell0 = np.zeros(self.ncase + 1, np.int32)
        self.bface0 = np.zeros(self.ncase + 1, np.int32)
        self._call("mfg_batch_layout", _lib.ptr(self.cell0, _lib.i32p),
                   _lib.ptr(self.bface0, _lib.i32p))
        self.n_cell = int(self.cell0[-1])
        self.n = self.n_cell + int(self.bface0[-1])

    def iterate(self, n: int, norms: bool = True) -> np.ndarray | None:
        """``n`` fused iterations of every case; norms shape ``[n, ncase, 5]``."""
        out = np.zeros(5 * n * self.ncase) if norms else None
        self._call("mfg_iterate", int(n), int(self.iter_done),
                   _lib.ptr(out) if norms else None)
        self.iter_done += n
        return out.reshape(n, self.ncase, 5) if norms else None

    def residual_norm(self) -> np.ndarray:
        out = np.zeros(5 * self.ncase)
        self._call("mfg_batch_residual_norm", _lib.ptr(out))
        return out.reshape(self.ncase, 5)

    @property
    def dt_extrema(self):
        out = np.zeros(2 * self.ncase)
        self._call("mfg_batch_dt_extrema", _lib.ptr(out))
        return [(out[2 * k], out[2 * k + 1]) for k in range(self.ncase)]

    def download(self, field: str) -> np.ndarray:
        """The union array (cells of all cases, then ghosts of all cases)."""
        C, n = self.n_cell, self.n
        size = {"q": 5 * n, "res": 5 * C, "dt": C, "dq": 5 * n, "dqdx": 5 * n, "dqdy": 5 * n,
                "dqdz": 5 * n, "diag": C, "limiter": 5 * C}[field]
        out = np.empty(size)
        self._call("mfg_download", _lib.FIELD[field], _lib.ptr(out))
        return out

    def split(self, field: str, arr: np.ndarray) -> list:
        """Per-case arrays, each in the single-case layout of its grid."""
        C, n = self.n_cell, self.n
        per_cell = field in ("res", "dt", "diag")
        nv = 1 if field in ("dt", "diag") else 5
        stride = C if per_cell else n
        out = []
        for k in range(self.ncase):
            a, b = int(self.cell0[k]), int(self.cell0[k + 1])
            ga, gb = C + int(self.bface0[k]), C + int(self.bface0[k + 1])
            parts = []
            for v in range(nv):
                base = v * stride
                parts.append(arr[base + a:base + b])
                if not per_cell:
                    parts.append(arr[base + ga:base + gb])
            out.append(np.concatenate(parts))
        return out

    def download_cases(self, field: str) -> list:
        return self.split(field, self.download(field))

    def upload_cases(self, qs):
        """Set the state of every case (each [5 n_k] in its own layout)."""
        C, n = self.n_cell, self.n
        q = np.empty(5 * n)
        for k, qk in enumerate(qs):
            a, b = int(self.cell0[k]), int(self.cell0[k + 1])
            ga, gb = C + int(self.bface0[k]), C + int(self.bface0[k + 1])
            nk = (b - a) + (gb - ga)
            qk = np.asarray(qk, np.float64).reshape(5, nk)
            for v in range(5):
                q[v * n + a:v * n + b] = qk[v, :b - a]
                q[v * n + ga:v * n + gb] = qk[v, b - a:]
        self.upload_q(q)


# Reference-named entry points (src/Kernels/*.h), operating on a Solver.# Reference-named entry points (src/Kernels/*.h), operating on a Solver.

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
