"""Build the mfgpu shared library in-tree (``minifs_b200/_lib/libmfgpu.so``).

``nvcc`` cross-compiles for sm_100a only; no GPU is needed to build.  The
device code is compiled with ``--fmad=false`` and the host code with
``-ffp-contract=off`` so that every floating-point operation rounds as in the
reference's plain x86-64 build (no fused multiply-adds anywhere).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libmfgpu.so")
INCLUDE = os.path.join(ROOT, "include")

SOURCES = ["mfg_device.cu", "mfg_prep.cu", "mfg_host.cpp", "mfg_io.cpp"]
DEPS = SOURCES + ["mfg_kernels.cuh", "mfg_internal.h"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise FileNotFoundError("nvcc not found")


def host_cxx() -> str:
    # the system driver (the one the reference's build uses)
    for cand in ("/usr/bin/g++", shutil.which("g++")):
        if cand and os.path.exists(cand):
            return cand
    raise FileNotFoundError("g++ not found")


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, s) for s in DEPS] + [os.path.join(INCLUDE, "mfgpu.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    tmp = LIB + ".tmp"
    cmd = [nvcc(), "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
           "-lineinfo", "--fmad=false", "-ccbin", host_cxx(),
           "-Xcompiler", "-fPIC,-ffp-contract=off,-O3", "-shared",
           "-I" + INCLUDE, "-I" + CSRC, "-o", tmp] + \
          [os.path.join(CSRC, s) for s in SOURCES] + ["-lcudart"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


SHIM = os.path.join(HERE, "shim")
DROPIN = os.path.join(SHIM, "_build", "minifs_dropin")


def reference_root() -> str:
    """The MiniFS source tree the oracle and the drop-in shim build against:
    the environment variable MINIFS_REF, else /root/reference."""
    return os.environ.get("MINIFS_REF", "/root/reference")


def build_dropin(ref: str | None = None, verbose: bool = False) -> str | None:
    """The reference's driver sequence on libmfgpu through the shim
    (``shim/mfgpu_shim.cpp`` in place of the reference's four kernel files,
    ``shim/dropin_main.cpp`` for main.cpp's hard-coded set-up), linked with
    the reference's unmodified ``src/Base`` and ``load_grid.cpp`` read in
    place (``ref``, default ``reference_root()``).  Built only where the
    reference sources exist; the binary finds libmfgpu.so next to the
    package through its run path."""
    src = os.path.join(ref or reference_root(), "src")
    if not os.path.isdir(src):
        return None
    os.makedirs(os.path.dirname(DROPIN), exist_ok=True)
    base = sorted(os.path.join(src, "Base", f) for f in os.listdir(os.path.join(src, "Base"))
                  if f.endswith(".cpp"))
    cmd = [host_cxx(), "-std=c++11", "-O3", "-ffp-contract=off", "-w", "-o", DROPIN,
           os.path.join(SHIM, "dropin_main.cpp"), os.path.join(SHIM, "mfgpu_shim.cpp")] + \
        base + [os.path.join(src, "Kernels", "load_grid.cpp"),
                "-I" + os.path.join(src, "Base"), "-I" + os.path.join(src, "Kernels"),
                "-I" + INCLUDE, "-L" + LIBDIR, "-lmfgpu", "-Wl,-rpath,$ORIGIN/../../_lib"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return DROPIN


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
