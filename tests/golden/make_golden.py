"""Regenerate the golden fixtures in this directory from the MiniFS reference.

Runs ``oracle/_ref/minifs_ref`` (serial build of the unmodified reference
sources, built by ``make -C oracle ref``) and ``minifs_ref_tdtree`` on small
seeded meshes and stores, per case, the inputs (mesh recipe and the sha256 of
the FlowStar file the reference read, or the mesh itself when it came out of
the reference's TDTree renumbering), the preprocessing arrays, and the
iteration outputs.  Usage:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from minifs_b200 import meshgen  # noqa: E402
from oracle import refrun  # noqa: E402

PARAM_NAMES = ["mach", "alpha", "beita", "re", "T", "gam", "gascon", "cfl_start", "cfl_end",
               "cfl_nstep", "lhs_omga", "alf_l", "ratio_dtmax", "amu", "ainf", "uqq", "u_s", "v_s",
               "w_s", "p_s", "rho_s", "p_bar", "gamm1", "p_stag", "e_stag", "p_min", "p_max",
               "rho_min", "rho_max", "p_break", "e_stag_max", "cfl_min", "cfl_ratio"]

PREP_KEYS = ["dims", "f2c", "nnpf", "f2n", "x", "y", "z", "xfn", "yfn", "zfn", "area", "xfc",
             "yfc", "zfc", "xcc", "ycc", "zcc", "vol", "bctype", "wnode", "nmark", "wbface",
             "nnpc", "c2n", "wc2n", "nodesymm", "xfn_n_symm", "yfn_n_symm", "zfn_n_symm",
             "params", "init.q", "init.dqdx"]

CASES = {
    # config-1 generator at a fixture-sized resolution: cube, far field
    "cube4": dict(mesh=dict(kind="box", nx=4, ny=4, nz=4, jitter=0.15, seed=7),
                  flow=dict(mach=0.5, alpha=2.0, cfl_start=10.0, cfl_end=10.0, bump_amp=0.05,
                            bump_sigma=0.1, bump_x0=0.5, bump_y0=0.5, bump_z0=0.5),
                  iters=12, dump="0,1,11"),
    # the channel generator: slip wall with a bump at the bottom
    "channel": dict(mesh=dict(kind="box", nx=8, ny=3, nz=3, lx=4.0, jitter=0.1, seed=5,
                              bc=[6, 6, 6, 6, 3, 6], bump=[0.05, 0.2, 1.5]),
                    flow=dict(mach=0.7, alpha=0.0, cfl_start=30.0, cfl_end=30.0, bump_amp=0.05,
                              bump_sigma=0.1, bump_x0=2.0, bump_y0=0.5, bump_z0=0.5),
                    iters=12, dump="0,11"),
    # CFL ramp (cfl_start != cfl_end, pow in LimitTimeStep), strong jitter
    "ramp5": dict(mesh=dict(kind="box", nx=5, ny=4, nz=3, jitter=0.2, seed=13),
                  flow=dict(mach=0.8, alpha=-3.0, beita=1.5, cfl_start=2.0, cfl_end=20.0,
                            cfl_nstep=6, bump_amp=0.1, bump_sigma=0.15, bump_x0=0.4,
                            bump_y0=0.5, bump_z0=0.6),
                  iters=10, dump="0,9"),
}
# the reference's own TDTree renumbering (METIS-based) of a cube mesh
TDTREE_CASE = dict(mesh=dict(kind="box", nx=8, ny=8, nz=8, jitter=0.15, seed=3),
                   flow=dict(mach=0.5, alpha=2.0, cfl_start=10.0, cfl_end=10.0, bump_amp=0.05,
                             bump_sigma=0.1, bump_x0=0.5, bump_y0=0.5, bump_z0=0.5),
                   iters=6, dump="5")


def build_mesh(spec: dict) -> meshgen.RawMesh:
    bump = tuple(spec["bump"]) if spec.get("bump") else None
    return meshgen.box_mesh(spec["nx"], spec["ny"], spec["nz"], lx=spec.get("lx", 1.0),
                            ly=spec.get("ly", 1.0), lz=spec.get("lz", 1.0),
                            jitter=spec["jitter"], seed=spec["seed"],
                            bc_types=tuple(spec.get("bc", [6] * 6)), bump=bump)


def mfl_sha256(mesh: meshgen.RawMesh) -> str:
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "g.mfl")
        meshgen.write_mfl(mesh, p)
        with open(p, "rb") as f:
            return hashlib.sha256(f.read()).hexdigest()


def save(name: str, case: dict, dump: dict, extra: dict, keep=None) -> None:
    out = {}
    for k in PREP_KEYS:
        out[k] = dump[k]
    for k, v in dump.items():
        if k.startswith("it") or k.startswith("final.") or k == "norms":
            if keep is None or k in keep:
                out[k] = v
    out.update(extra)
    meta = dict(case=case, param_names=PARAM_NAMES)
    out["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **out)
    print(f"{path}: {os.path.getsize(path) / 1024:.0f} KiB")


def main() -> None:
    if not refrun.available():
        sys.exit("oracle/_ref/minifs_ref is not built: make -C oracle ref")
    for name, case in CASES.items():
        mesh = build_mesh(case["mesh"])
        flow = dict(case["flow"], n_steps=case["iters"])
        r = refrun.run(mesh, flow, dump_iters=case["dump"])
        save(name, case, r, {"mfl_sha256": np.frombuffer(mfl_sha256(mesh).encode(), np.uint8)})
    case = TDTREE_CASE
    mesh = build_mesh(case["mesh"])
    flow = dict(case["flow"], n_steps=case["iters"])
    td = refrun.run(mesh, flow, tdtree=True, write_mesh=True, threads=1, dump_iters=case["dump"])
    ren = meshgen.read_mfl(td["renumbered_mfl"])
    ren.patches = mesh.patches
    # the serial reference on the renumbered grid: the plain-parity target
    r = refrun.run(ren, flow, dump_iters=case["dump"])
    # the grid itself is x, y, z, nnpf, f2n of the dump plus the file's f2c
    extra = {"raw.f2c": _raw_f2c(td["renumbered_mfl"]), "tdtree.final.q": td["final.q"],
             "tdtree.norms": td["norms"]}
    save("tdtree8", case, r, extra,
         keep={"norms", "final.q", "final.res", "final.dqdx", "final.dt_extrema"})


def _raw_f2c(path: str) -> np.ndarray:
    """f2c exactly as stored in the file (before the reader's boundary flip)."""
    with open(path, "rb") as f:
        hdr = np.frombuffer(f.read(12), np.int32)
        nn, nf = int(hdr[0]), int(hdr[1])
        f.seek(12 + 24 * nn)
        nnpf = np.frombuffer(f.read(4 * nf), np.int32)
        f.seek(12 + 24 * nn + 4 * nf + 4 * int(nnpf.sum()))
        return np.frombuffer(f.read(8 * nf), np.int32).copy()


if __name__ == "__main__":
    main()
