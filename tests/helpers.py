"""Shared test helpers: golden fixtures, oracle and product solvers on the
same inputs, and comparisons."""
from __future__ import annotations

import json
import os

import numpy as np

from minifs_b200 import meshgen

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
PARAM_NAMES = ["mach", "alpha", "beita", "re", "T", "gam", "gascon", "cfl_start", "cfl_end",
               "cfl_nstep", "lhs_omga", "alf_l", "ratio_dtmax", "amu", "ainf", "uqq", "u_s", "v_s",
               "w_s", "p_s", "rho_s", "p_bar", "gamm1", "p_stag", "e_stag", "p_min", "p_max",
               "rho_min", "rho_max", "p_break", "e_stag_max", "cfl_min", "cfl_ratio"]
GOLDEN_CASES = ("cube4", "channel", "ramp5")


def load_golden(name: str) -> dict:
    with np.load(os.path.join(GOLDEN, f"{name}.npz")) as z:
        d = {k: z[k] for k in z.files}
    d["meta"] = json.loads(bytes(d["meta"]).decode())
    return d


def golden_params(d: dict) -> dict:
    p = dict(zip(PARAM_NAMES, (float(v) for v in d["params"])))
    p["cfl_nstep"] = int(p["cfl_nstep"])
    return p


def build_mesh(spec: dict) -> meshgen.RawMesh:
    bump = tuple(spec["bump"]) if spec.get("bump") else None
    return meshgen.box_mesh(spec["nx"], spec["ny"], spec["nz"], lx=spec.get("lx", 1.0),
                            ly=spec.get("ly", 1.0), lz=spec.get("lz", 1.0),
                            jitter=spec["jitter"], seed=spec["seed"],
                            bc_types=tuple(spec.get("bc", [6] * 6)), bump=bump)


def raw_mesh_from_golden(d: dict) -> meshgen.RawMesh:
    """The grid a golden case ran on, as a raw (file-layout) mesh."""
    spec = d["meta"]["case"]["mesh"]
    if "raw.f2c" in d:  # renumbered by the reference's TDTree code
        m = meshgen.RawMesh(x=d["x"], y=d["y"], z=d["z"], nnpf=d["nnpf"], f2n=d["f2n"],
                            f2c=d["raw.f2c"].copy(), n_cell=int(d["dims"][2]),
                            n_bface=int(d["dims"][3]))
    else:
        m = build_mesh(spec)
    m.patches = [(i + 1, t) for i, t in enumerate(spec.get("bc", [6] * 6))]
    return m


def make_product_params(d: dict):
    from minifs_b200 import grid as gr
    flow = d["meta"]["case"]["flow"]
    return gr.make_params(mach=flow["mach"], alpha=flow["alpha"], beita=flow.get("beita", 0.0),
                          cfl_start=flow["cfl_start"], cfl_end=flow["cfl_end"],
                          cfl_nstep=flow.get("cfl_nstep", 2000))


def prepare_product(d: dict):
    """Run the product's host preprocessing on the golden case's mesh."""
    from minifs_b200 import grid as gr
    flow = d["meta"]["case"]["flow"]
    p = make_product_params(d)
    pg = gr.prepare(raw_mesh_from_golden(d), p, bump_amp=flow["bump_amp"],
                    bump_sigma=flow["bump_sigma"],
                    bump_center=(flow["bump_x0"], flow["bump_y0"], flow["bump_z0"]))
    return pg, p


def oracle_from(arrays: dict, params: dict, q0, dims):
    from oracle import oracle_py
    return oracle_py.OracleSolver(arrays, params, q0, dims)


def assert_bitwise(a, b, what=""):
    a = np.asarray(a)
    b = np.asarray(b)
    assert a.shape == b.shape, f"{what}: shape {a.shape} != {b.shape}"
    if not np.array_equal(a, b):
        bad = np.nonzero(a != b)[0]
        i = int(bad[0])
        rel = np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)
        raise AssertionError(f"{what}: {bad.size} entries differ, first at {i}: "
                             f"{a[i]!r} vs {b[i]!r}; max rel {rel:.3e}")
