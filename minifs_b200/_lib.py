"""ctypes binding of ``libmfgpu.so`` (declarations in include/mfgpu.h).

Loading fails loudly when the library is missing: there is no fallback
implementation of the hot path.
"""
from __future__ import annotations

import ctypes as ct
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libmfgpu.so")

i32p = ct.POINTER(ct.c_int32)
f64p = ct.POINTER(ct.c_double)

MFG_OK = 0
ERRORS = {-1: "invalid argument", -2: "CUDA error", -3: "out of memory",
          -4: "device wait timed out", -5: "non-finite value", -6: "unsupported configuration",
          -7: "bad mesh", -8: "no usable CUDA device",
          -9: "file missing, truncated or malformed"}

FIELD = {"q": 0, "res": 1, "dt": 2, "dq": 3, "dqdx": 4, "dqdy": 5, "dqdz": 6, "diag": 7,
         "limiter": 8}
PREC = {"fp64": 0, "mixed": 1}
PHASES = ("face_gather", "sweep_fwd", "sweep_bwd_update", "node_values", "grad_faces", "norm")

PARAM_INPUTS = ("mach", "alpha", "beita", "re", "T", "gam", "gascon", "cfl_start", "cfl_end")
PARAM_FIELDS = (
    [(k, ct.c_double) for k in PARAM_INPUTS] + [("cfl_nstep", ct.c_int32)] +
    [(k, ct.c_double) for k in ("lhs_omga", "epsa_r", "ratio_dtmax", "amu", "ainf", "uqq",
                                "u_s", "v_s", "w_s", "p_s", "rho_s", "p_bar", "gamm1", "p_stag",
                                "e_stag", "p_min", "p_max", "rho_min", "rho_max", "p_break",
                                "e_stag_max", "cfl_min", "cfl_ratio", "alf_l")])


class Params(ct.Structure):
    _fields_ = PARAM_FIELDS

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


MESH_I32 = ("f2c", "nnpf", "f2n", "bctype")
MESH_F64_FACE = ("xfn", "yfn", "zfn", "area", "xfc", "yfc", "zfc")
MESH_F64_CELL = ("xcc", "ycc", "zcc", "vol")


class Mesh(ct.Structure):
    _fields_ = ([("n_node", ct.c_int32), ("n_face", ct.c_int32), ("n_cell", ct.c_int32),
                 ("n_bface", ct.c_int32)] +
                [(k, i32p) for k in MESH_I32] +
                [(k, f64p) for k in MESH_F64_FACE + MESH_F64_CELL] +
                [("wnode", f64p), ("nmark", i32p), ("wbface", f64p), ("nnpc", i32p),
                 ("c2n", i32p), ("wc2n", f64p), ("nodesymm", i32p), ("xfn_n_symm", f64p),
                 ("yfn_n_symm", f64p), ("zfn_n_symm", f64p), ("lusgs_order", i32p),
                 ("lusgs_layer", i32p)])


class Info(ct.Structure):
    _fields_ = [("n_cell", ct.c_int32), ("n_face", ct.c_int32), ("n_node", ct.c_int32),
                ("n_bface", ct.c_int32), ("fw_levels", ct.c_int32), ("bw_levels", ct.c_int32),
                ("max_level_cells", ct.c_int32), ("precision", ct.c_int32),
                ("device_bytes", ct.c_int64), ("sweep_mode", ct.c_int32),
                ("graph_ready", ct.c_int32), ("ncase", ct.c_int32),
                ("sweep_chunks", ct.c_int32), ("sweep_lanes", ct.c_int32),
                ("sweep_records", ct.c_int32), ("sweep_chunking", ct.c_int32),
                ("sweep_ring_records", ct.c_int32 * 2), ("sweep_global_records", ct.c_int32 * 2),
                ("sweep_cross_records", ct.c_int32 * 2), ("sweep_model_us", ct.c_double * 2),
                ("sweep_kernel", ct.c_int32)]


TUNE_KNOBS, TUNE_CANDS = 8, 4
KNOBS = {0: "sweep_kernel", 1: "sweep_chunking", 2: "sweep_mode", 3: "face_gather_blocks_per_sm",
         4: "face_flux_blocks_per_sm", 5: "node_values_block", 6: "grad_faces_block",
         7: "gather_lanes_per_cell"}


class TuneReport(ct.Structure):
    _fields_ = [("n_knobs", ct.c_int32), ("knob", ct.c_int32 * TUNE_KNOBS),
                ("n_cand", ct.c_int32 * TUNE_KNOBS),
                ("cand", (ct.c_int32 * TUNE_CANDS) * TUNE_KNOBS),
                ("ms", (ct.c_double * TUNE_CANDS) * TUNE_KNOBS),
                ("chosen", ct.c_int32 * TUNE_KNOBS), ("ms_initial", ct.c_double),
                ("ms_final", ct.c_double)]


class RawGrid(ct.Structure):
    _fields_ = [("n_node", ct.c_int32), ("n_face", ct.c_int32), ("n_cell", ct.c_int32),
                ("n_bface", ct.c_int32), ("x", f64p), ("y", f64p), ("z", f64p),
                ("nnpf", i32p), ("f2n", i32p), ("f2c", i32p)]


class Mfl(ct.Structure):
    _fields_ = [("n_node", ct.c_int32), ("n_face", ct.c_int32), ("n_cell", ct.c_int32),
                ("n_bface", ct.c_int32), ("x", f64p), ("y", f64p), ("z", f64p),
                ("nnpf", i32p), ("f2n", i32p), ("f2c", i32p),
                ("n_iface", ct.c_int32), ("nbz", i32p), ("nbf", i32p),
                ("n_inode", ct.c_int32), ("nbsn", i32p), ("nbzn", i32p), ("nbrn", i32p)]


class Halo(ct.Structure):
    _fields_ = [("n_send", ct.c_int32), ("send_cells", i32p), ("n_recv", ct.c_int32),
                ("recv_bfaces", i32p), ("n_node", ct.c_int32), ("nodes", i32p),
                ("send_rows", ct.c_void_p), ("recv_rows", ct.c_void_p),
                ("node_send", ct.c_void_p), ("node_recv", ct.c_void_p),
                ("ext", ct.c_void_p), ("norm_sq", ct.c_void_p),
                ("grad_send", ct.c_void_p), ("grad_recv", ct.c_void_p)]


# mfg_halo_phase phases
HALO = {"pack_q": 0, "face": 1, "forward": 2, "backward": 3, "nodes": 4, "gradient": 5,
        "check": 6, "limit": 7}


class MfgError(RuntimeError):
    def __init__(self, func: str, code: int, detail: str = ""):
        msg = f"{func} failed: {ERRORS.get(code, code)}"
        if detail:
            msg += f" ({detail})"
        super().__init__(msg)
        self.code = code


_lib = None


def load(build_if_missing: bool = True):
    """Load libmfgpu.so, building it in-tree with nvcc if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        if not build_if_missing:
            raise FileNotFoundError(f"{LIB_PATH} is not built (python -m minifs_b200.build)")
        from . import build as _build
        _build.build()
    lib = ct.CDLL(LIB_PATH)
    ctxp = ct.c_void_p
    sig = {
        "mfg_params_default": (None, [ct.POINTER(Params)]),
        "mfg_params_derive": (ct.c_int, [ct.POINTER(Params)]),
        "mfg_create": (ct.c_int, [ct.POINTER(Mesh), ct.POINTER(Params), f64p, ct.c_int32,
                                  ct.c_int32, ct.POINTER(ctxp)]),
        "mfg_create_batch": (ct.c_int, [ct.c_int32, ct.POINTER(Mesh), ct.POINTER(Params),
                                        ct.POINTER(f64p), ct.c_int32, ct.c_int32,
                                        ct.POINTER(ctxp)]),
        "mfg_batch_layout": (ct.c_int, [ctxp, i32p, i32p]),
        "mfg_batch_dt_extrema": (ct.c_int, [ctxp, f64p]),
        "mfg_batch_residual_norm": (ct.c_int, [ctxp, f64p]),
        "mfg_destroy": (ct.c_int, [ctxp]),
        "mfg_set_stream": (ct.c_int, [ctxp, ct.c_void_p]),
        "mfg_set_params": (ct.c_int, [ctxp, ct.POINTER(Params)]),
        "mfg_info_get": (ct.c_int, [ctxp, ct.POINTER(Info)]),
        "mfg_set_sweep_mode": (ct.c_int, [ctxp, ct.c_int32]),
        "mfg_set_sweep_lanes": (ct.c_int, [ctxp, ct.c_int32]),
        "mfg_set_gather_lanes": (ct.c_int, [ctxp, ct.c_int32]),
        "mfg_set_chunking": (ct.c_int, [ct.c_int32]),
        "mfg_plan_chunks": (ct.c_int, [ct.c_int32, ct.c_int32, i32p, i32p, i32p, i32p, f64p, f64p,
                                       f64p, ct.c_int32, ct.c_int32, ct.c_int32, i32p, i32p,
                                       f64p]),
        "mfg_set_sweep_kernel": (ct.c_int, [ct.c_int32]),
        "mfg_autotune_sweeps": (ct.c_int, [ctxp, ct.c_int32, ct.c_int32, f64p]),
        "mfg_autotune": (ct.c_int, [ctxp, ct.c_int32, ct.c_int32, ct.c_int32,
                                    ct.POINTER(TuneReport)]),
        "mfg_selftest_sweep_timeout": (ct.c_int, [ctxp, ct.c_int64]),
        "mfg_selftest_division": (ct.c_int, [ct.c_int64, ct.c_uint64,
                                             ct.POINTER(ct.c_int64)]),
        "mfg_selftest_functions": (ct.c_int, [ct.c_int32, ct.c_int32, f64p, f64p, f64p]),
        "mfg_selftest_division_fast": (ct.c_int, [ct.c_int64, ct.c_uint64,
                                                  ct.POINTER(ct.c_int64)]),
        "mfg_zero_residuals": (ct.c_int, [ctxp]),
        "mfg_inviscid_flux": (ct.c_int, [ctxp]),
        "mfg_compute_timestep": (ct.c_int, [ctxp, ct.c_int32]),
        "mfg_forward_lusgs": (ct.c_int, [ctxp]),
        "mfg_calculate_gradient": (ct.c_int, [ctxp]),
        "mfg_set_ghost_variables": (ct.c_int, [ctxp]),
        "mfg_set_live_bc": (ct.c_int, [ctxp, ct.c_int32]),
        "mfg_set_flux_fp64": (ct.c_int, [ctxp, ct.c_int32]),
        "mfg_set_order": (ct.c_int, [ctxp, ct.c_int32, ct.c_double]),
        "mfg_iterate": (ct.c_int, [ctxp, ct.c_int32, ct.c_int32, f64p]),
        "mfg_iterate_host": (ct.c_int, [ctxp, ct.c_int32, ct.c_int32, f64p, f64p, f64p, f64p]),
        "mfg_residual_norm": (ct.c_int, [ctxp, f64p]),
        "mfg_profile_phases": (ct.c_int, [ctxp, ct.c_int32, ct.c_int32, f64p]),
        "mfg_residual_norm_static": (ct.c_int, [ct.c_void_p, ct.c_int32, ct.c_void_p,
                                                ct.c_void_p]),
        "mfg_get_dt_extrema": (ct.c_int, [ctxp, f64p, f64p]),
        "mfg_set_dt_extrema": (ct.c_int, [ctxp, ct.c_double, ct.c_double]),
        "mfg_halo_set": (ct.c_int, [ctxp, ct.POINTER(Halo)]),
        "mfg_halo_phase": (ct.c_int, [ctxp, ct.c_int32, ct.c_int32]),
        "mfg_download": (ct.c_int, [ctxp, ct.c_int32, f64p]),
        "mfg_upload": (ct.c_int, [ctxp, ct.c_int32, f64p]),
        "mfg_sync": (ct.c_int, [ctxp]),
        "mfg_error_string": (ct.c_char_p, [ct.c_int32]),
        "mfg_last_cuda_error": (ct.c_char_p, []),
        "mfg_kernel_launches": (ct.c_int64, []),
        "mfg_prep_specify_bc": (ct.c_int, [ct.POINTER(RawGrid), ct.c_int32, i32p, i32p]),
        "mfg_prep_metrics": (ct.c_int, [ct.POINTER(RawGrid)] + [f64p] * 11),
        "mfg_prep_init_flow": (ct.c_int, [ct.POINTER(RawGrid), ct.POINTER(Params), i32p] +
                               [f64p] * 6 + [ct.c_double] * 5 + [f64p]),
        "mfg_prep_c2n_size": (ct.c_int, [ct.POINTER(RawGrid), ct.POINTER(ct.c_int64)]),
        "mfg_prep_node_weights": (ct.c_int, [ct.POINTER(RawGrid), i32p] + [f64p] * 9 +
                                  [f64p, i32p, f64p, i32p, i32p, f64p, i32p, f64p, f64p, f64p]),
        "mfg_prep_gpu_run": (ct.c_int, [ct.POINTER(RawGrid), i32p, ct.c_int32,
                                        ct.POINTER(ct.c_void_p)]),
        "mfg_prep_gpu_c2n_size": (ct.c_int, [ct.c_void_p, ct.POINTER(ct.c_int64)]),
        "mfg_prep_gpu_kernel_ms": (ct.c_int, [ct.c_void_p, f64p]),
        "mfg_prep_gpu_metrics": (ct.c_int, [ct.c_void_p] + [f64p] * 11),
        "mfg_prep_gpu_node_weights": (ct.c_int, [ct.c_void_p, f64p, i32p, f64p, i32p, i32p, f64p,
                                                 i32p, f64p, f64p, f64p]),
        "mfg_prep_gpu_destroy": (ct.c_int, [ct.c_void_p]),
        "mfg_prep_gpu_init_flow": (ct.c_int, [ct.c_void_p, ct.POINTER(Params)] +
                                   [ct.c_double] * 5 + [f64p]),
        "mfg_create_from_prep": (ct.c_int, [ct.c_void_p, ct.POINTER(Params), f64p, ct.c_int32,
                                            ct.POINTER(ctxp)]),
        "mfg_mfl_read": (ct.c_int, [ct.c_char_p, ct.POINTER(ct.POINTER(Mfl))]),
        "mfg_mfl_write": (ct.c_int, [ct.c_char_p, ct.POINTER(Mfl)]),
        "mfg_mfl_free": (ct.c_int, [ct.POINTER(Mfl)]),
        "mfg_bc_read": (ct.c_int, [ct.c_char_p, ct.c_int32, i32p, i32p, i32p]),
        "mfg_bc_write": (ct.c_int, [ct.c_char_p, ct.c_int32, i32p, i32p]),
        "mfg_checkpoint_write": (ct.c_int, [ct.c_char_p, ct.c_int64, ct.c_int64, ct.c_int32,
                                            ct.c_double, ct.c_double, f64p]),
        "mfg_checkpoint_read": (ct.c_int, [ct.c_char_p, ct.c_int64, ct.c_int64,
                                           ct.POINTER(ct.c_int32), f64p, f64p, f64p]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(func: str, code: int) -> None:
    if code != MFG_OK:
        detail = ""
        if code == -2 and _lib is not None:
            detail = _lib.mfg_last_cuda_error().decode(errors="replace")
        raise MfgError(func, code, detail)


def ptr(a: np.ndarray, kind=f64p):
    return a.ctypes.data_as(kind)


def kernel_launches() -> int:
    return int(load().mfg_kernel_launches())
