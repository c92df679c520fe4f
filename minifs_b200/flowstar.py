"""FlowStar grid (``.mfl``) and boundary-condition (``bc.para``) files
through the library's C reader and writer (``mfg_mfl_*``, ``mfg_bc_*``).

``read_case`` gives the raw mesh ``grid.prepare`` takes, the way the
reference's ``ReadMFlowGrid_binary`` and ``ReadMFlowBoundaryCondition``
(src/Kernels/load_grid.cpp:129-314) leave it: faces with a boundary on the
left flipped, boundary faces counted, the patch table in file order.
"""
from __future__ import annotations

import ctypes as ct
import os
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .meshgen import RawMesh


@dataclass
class Interfaces:
    """Interface block of a partitioned grid file: per interface face the
    zone of its other side and its face there; per interface node its own
    index, the zone and its index there."""
    nbz: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    nbf: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    nbsn: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    nbzn: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    nbrn: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))


def _path(p) -> bytes:
    return os.fsencode(os.fspath(p))


def read_grid(path) -> tuple[RawMesh, Interfaces]:
    lib = _lib.load()
    out = ct.POINTER(_lib.Mfl)()
    _lib.check("mfg_mfl_read", lib.mfg_mfl_read(_path(path), ct.byref(out)))
    try:
        g = out.contents

        def arr(p, n, dt):
            if n == 0:
                return np.zeros(0, dt)
            return np.ctypeslib.as_array(p, shape=(n,)).astype(dt, copy=True)

        N, F = g.n_node, g.n_face
        L = int(arr(g.nnpf, F, np.int64).sum())
        mesh = RawMesh(x=arr(g.x, N, np.float64), y=arr(g.y, N, np.float64),
                       z=arr(g.z, N, np.float64), nnpf=arr(g.nnpf, F, np.int32),
                       f2n=arr(g.f2n, L, np.int32), f2c=arr(g.f2c, 2 * F, np.int32),
                       n_cell=g.n_cell, n_bface=g.n_bface, patches=[])
        itf = Interfaces(nbz=arr(g.nbz, g.n_iface, np.int32), nbf=arr(g.nbf, g.n_iface, np.int32),
                         nbsn=arr(g.nbsn, g.n_inode, np.int32),
                         nbzn=arr(g.nbzn, g.n_inode, np.int32),
                         nbrn=arr(g.nbrn, g.n_inode, np.int32))
    finally:
        lib.mfg_mfl_free(out)
    return mesh, itf


def write_grid(mesh: RawMesh, path, interfaces: Interfaces | None = None) -> None:
    lib = _lib.load()
    itf = interfaces or Interfaces()
    keep = []

    def a(x, dt, kind):
        v = np.ascontiguousarray(x, dt)
        keep.append(v)
        return _lib.ptr(v, kind)

    g = _lib.Mfl()
    g.n_node, g.n_face, g.n_cell, g.n_bface = mesh.n_node, mesh.n_face, mesh.n_cell, mesh.n_bface
    g.x, g.y, g.z = (a(v, np.float64, _lib.f64p) for v in (mesh.x, mesh.y, mesh.z))
    g.nnpf = a(mesh.nnpf, np.int32, _lib.i32p)
    g.f2n = a(mesh.f2n, np.int32, _lib.i32p)
    g.f2c = a(mesh.f2c, np.int32, _lib.i32p)
    if len(itf.nbz) != len(itf.nbf) or not (len(itf.nbsn) == len(itf.nbzn) == len(itf.nbrn)):
        raise ValueError("interface arrays of one block must have equal lengths")
    g.n_iface, g.n_inode = len(itf.nbz), len(itf.nbsn)
    g.nbz, g.nbf = a(itf.nbz, np.int32, _lib.i32p), a(itf.nbf, np.int32, _lib.i32p)
    g.nbsn, g.nbzn, g.nbrn = (a(v, np.int32, _lib.i32p) for v in (itf.nbsn, itf.nbzn, itf.nbrn))
    _lib.check("mfg_mfl_write", lib.mfg_mfl_write(_path(path), ct.byref(g)))


def read_bc(path, cap: int = 4096) -> list[tuple[int, int]]:
    lib = _lib.load()
    n = ct.c_int32(0)
    pid = np.zeros(cap, np.int32)
    typ = np.zeros(cap, np.int32)
    _lib.check("mfg_bc_read", lib.mfg_bc_read(_path(path), cap, ct.byref(n),
                                              _lib.ptr(pid, _lib.i32p), _lib.ptr(typ, _lib.i32p)))
    return [(int(pid[i]), int(typ[i])) for i in range(n.value)]


def write_bc(patches, path) -> None:
    lib = _lib.load()
    pid = np.array([p for p, _ in patches], np.int32)
    typ = np.array([t for _, t in patches], np.int32)
    _lib.check("mfg_bc_write", lib.mfg_bc_write(_path(path), len(patches),
                                                _lib.ptr(pid, _lib.i32p),
                                                _lib.ptr(typ, _lib.i32p)))


def read_case(grid_path, bc_path) -> RawMesh:
    """A grid file and its bc.para as one raw mesh (interfaces dropped)."""
    mesh, _ = read_grid(grid_path)
    mesh.patches = read_bc(bc_path)
    return mesh
