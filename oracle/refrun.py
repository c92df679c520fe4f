"""TEST INFRASTRUCTURE ONLY: run the compiled MiniFS reference (oracle/_ref).

Only the tests, ``__graft_entry__.smoke`` and the CPU-baseline leg of
``bench.py`` import this module.  It writes a case (FlowStar ``.mfl`` grid,
``bc.para`` and a parameter file) into a scratch directory, runs
``oracle/_ref/minifs_ref`` (serial) or ``minifs_ref_tdtree`` (TDTree +
OpenMP) built by ``oracle/Makefile`` from the unmodified reference sources,
and parses the tagged binary dump written by ``oracle/ref_harness.cpp``.
"""
from __future__ import annotations

import json
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
SERIAL = os.path.join(REF_DIR, "minifs_ref")
TDTREE = os.path.join(REF_DIR, "minifs_ref_tdtree")

PARAM_KEYS = ("mach", "alpha", "beita", "re", "T", "gam", "gascon", "cfl_start", "cfl_end",
              "cfl_nstep", "n_steps", "lhs_omga", "epsa_r", "ratio_dtmax", "bump_amp",
              "bump_sigma", "bump_x0", "bump_y0", "bump_z0")


def available(tdtree: bool = False) -> bool:
    path = TDTREE if tdtree else SERIAL
    return os.path.isfile(path) and os.access(path, os.X_OK)


def read_dump(path: str) -> dict:
    """Parse an ``MFDUMP01`` file into ``{name: ndarray}``."""
    with open(path, "rb") as f:
        buf = f.read()
    if buf[:8] != b"MFDUMP01":
        raise ValueError(f"{path}: not a harness dump")
    out = {}
    off = 8
    while off < len(buf):
        ln = int(np.frombuffer(buf, np.int32, 1, off)[0]); off += 4
        name = buf[off:off + ln].decode(); off += ln
        code = chr(buf[off]); off += 1
        cnt = int(np.frombuffer(buf, np.int64, 1, off)[0]); off += 8
        dt = np.float64 if code == "d" else np.int32
        arr = np.frombuffer(buf, dt, cnt, off).copy()
        off += arr.nbytes
        out[name] = arr
    return out


def write_params(path: str, params: dict) -> None:
    with open(path, "w") as f:
        for k, v in params.items():
            if k not in PARAM_KEYS:
                raise KeyError(f"unknown harness parameter {k}")
            f.write(f"{k} {float(v)!r}\n")


def run(mesh, params: dict, *, tdtree: bool = False, dump_iters="0", threads: int | None = None,
        write_mesh: bool = False, workdir: str | None = None, dump: bool = True,
        timeout: float | None = None, light: bool = False, live_bc: bool = False) -> dict:
    """Run the reference on ``mesh`` (a ``meshgen.RawMesh``) and return the dump.

    The returned dict also carries ``"summary"`` (the JSON line the harness
    prints) and, with ``write_mesh``, ``"renumbered_mfl"`` (the path of the
    grid after the reference's own TDTree renumbering).
    """
    from minifs_b200 import meshgen

    exe = TDTREE if tdtree else SERIAL
    if not available(tdtree):
        raise FileNotFoundError(f"{exe} is not built (make -C oracle ref)")
    tmp = workdir or tempfile.mkdtemp(prefix="mfref_")
    mfl = os.path.join(tmp, "grid.mfl")
    bcp = os.path.join(tmp, "bc.para")
    par = os.path.join(tmp, "params.txt")
    out = os.path.join(tmp, "dump.bin")
    meshgen.write_mfl(mesh, mfl)
    meshgen.write_bc(mesh, bcp)
    write_params(par, params)
    cmd = [exe, "--mesh", mfl, "--bc", bcp, "--params", par]
    if dump or light:
        cmd += ["--out", out, "--dump-iters", str(dump_iters) if dump else "-1"]
    if light:
        cmd += ["--light"]
    if live_bc:
        cmd += ["--live-bc"]
    ren = os.path.join(tmp, "renumbered.mfl")
    if write_mesh:
        cmd += ["--write-mesh", ren]
    env = dict(os.environ)
    if threads is not None:
        env["OMP_NUM_THREADS"] = str(threads)
    proc = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=timeout)
    if proc.returncode != 0:
        raise RuntimeError(f"reference run failed ({proc.returncode}):\n{proc.stdout[-2000:]}\n"
                           f"{proc.stderr[-2000:]}")
    summary = None
    for line in proc.stdout.splitlines():
        line = line.strip()
        if line.startswith("{") and line.endswith("}"):
            summary = json.loads(line)
    res = read_dump(out) if (dump or light) else {}
    res["summary"] = summary
    res["stdout"] = proc.stdout
    if write_mesh:
        res["renumbered_mfl"] = ren
    return res
