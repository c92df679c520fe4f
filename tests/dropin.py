"""Runs the reference's driver sequence on libmfgpu through the drop-in shim
(minifs_b200/shim/_build/minifs_dropin) on a case written the way the
reference reads it; the dump has the reference harness's format."""
import os
import subprocess
import tempfile

from minifs_b200 import build, meshgen
from oracle import refrun


def available() -> bool:
    return os.path.isfile(build.DROPIN) and os.access(build.DROPIN, os.X_OK)


def run(mesh, params: dict, sync_every_call: bool = True, timeout: float = 600):
    tmp = tempfile.mkdtemp(prefix="mfdropin_")
    paths = {k: os.path.join(tmp, f) for k, f in
             (("mesh", "grid.mfl"), ("bc", "bc.para"), ("params", "params.txt"),
              ("out", "dump.bin"))}
    meshgen.write_mfl(mesh, paths["mesh"])
    meshgen.write_bc(mesh, paths["bc"])
    refrun.write_params(paths["params"], params)
    env = dict(os.environ)
    if sync_every_call:
        env["MFGPU_SYNC_EVERY_CALL"] = "1"
    cmd = [build.DROPIN] + [a for k in ("mesh", "bc", "params", "out")
                            for a in (f"--{k}", paths[k])]
    proc = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=timeout)
    res = {"returncode": proc.returncode, "stdout": proc.stdout, "stderr": proc.stderr}
    if proc.returncode == 0:
        res.update(refrun.read_dump(paths["out"]))
    return res
