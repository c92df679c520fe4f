"""Seeded tetrahedral box meshes in the FlowStar face-based layout.

The reference reads meshes of this layout in ``ReadMFlowGrid_binary``
(src/Kernels/load_grid.cpp:129-273): node coordinates, nodes per face,
face->node lists, and face->cell pairs where a boundary face carries the
negated patch id in its second slot.  Every consumer downstream assumes:

* the boundary faces are the first ``nBFace`` faces (load_grid.cpp:196-230,
  all kernels loop ``[0, nBFace)`` then ``[nBFace, nTFace)``);
* the face normal given by the node order points out of the first cell, or
  ``CellVolCentroid`` finds a negative volume and exits
  (src/Base/grid_polyhedra_auxiliary_functions.cpp:458-536).

The generator splits an ``nx*ny*nz`` hex block into six Kuhn tetrahedra per
hex (all sharing the hex's main diagonal, which makes the split conforming
across hexes), jitters the nodes with a counter-based splitmix64 stream, and
emits faces in a fixed, documented order:

* cells: ``6*hex + perm`` with ``hex = i + nx*(j + ny*k)``;
* boundary faces first, sorted by (cell, local slot); interior faces next,
  sorted by (lower cell, higher cell), with ``c1 = lower cell``.

Everything here is integer work or IEEE double arithmetic without libm
transcendental calls except ``math.exp`` for the wall bump (glibc, the same
library the reference links), so a mesh is bit-identical wherever it is
generated on this image.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# Boundary-condition type codes (src/Base/constant.h:47-51).
WALL = 3
SYMM = 4
FAR_FIELD = 6
FAR_FIELD_MOD = 61
INTERFACE = 10

# The six axis permutations (a, b, c); tet p of a hex walks e_a, e_b, e_c
# from the hex's low corner to its high corner.
PERMS = ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0))
_PERM_INDEX = {p: i for i, p in enumerate(PERMS)}

_MASK64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(x: np.ndarray) -> np.ndarray:
    """Vectorised splitmix64 finaliser over a uint64 counter array."""
    z = (x + np.uint64(0x9E3779B97F4A7C15)) & _MASK64
    z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & _MASK64
    z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & _MASK64
    return z ^ (z >> np.uint64(31))


def uniform01(seed: int, counters: np.ndarray) -> np.ndarray:
    """Doubles in [0, 1) from stream ``seed`` at the given counters (53-bit)."""
    base = splitmix64(np.full(1, seed, dtype=np.uint64))[0]
    with np.errstate(over="ignore"):
        bits = splitmix64(counters.astype(np.uint64) ^ base)
    return (bits >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


@dataclass
class RawMesh:
    """A mesh as stored in a FlowStar ``.mfl`` file plus its ``bc.para`` table.

    ``f2c`` holds ``(c1, c2)`` pairs; for a boundary face ``c2 = -patch_id``.
    ``patches`` maps patch id (1-based, file order) to a BC type code.
    """

    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    nnpf: np.ndarray
    f2n: np.ndarray
    f2c: np.ndarray
    n_cell: int
    n_bface: int
    patches: list = field(default_factory=list)

    @property
    def n_node(self) -> int:
        return int(self.x.shape[0])

    @property
    def n_face(self) -> int:
        return int(self.nnpf.shape[0])


def _node_id(i, j, k, nx, ny):
    return i + (nx + 1) * (j + (ny + 1) * k)


def _box_nodes(nx: int, ny: int, nz: int, lx: float, ly: float, lz: float, jitter: float,
               seed: int, bump):
    """Node coordinates of an ``nx*ny*nz`` hex block: node
    ``i + (nx+1)*(j + (ny+1)*k)``, interior coordinates jittered by up to
    ``jitter`` local spacings, the optional bottom bump (see ``box_mesh``)."""
    nx, ny, nz = int(nx), int(ny), int(nz)
    nn = (nx + 1) * (ny + 1) * (nz + 1)
    ii, jj, kk = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1),
                             np.arange(nz + 1), indexing="ij")
    # node id = i + (nx+1)*(j + (ny+1)*k): flatten in Fortran order of (i,j,k)
    ii = ii.ravel(order="F").astype(np.int64)
    jj = jj.ravel(order="F").astype(np.int64)
    kk = kk.ravel(order="F").astype(np.int64)
    node_ids = np.arange(nn, dtype=np.int64)
    coords = []
    for axis, (idx, n, length) in enumerate(((ii, nx, lx), (jj, ny, ly), (kk, nz, lz))):
        h = length / n
        c = idx.astype(np.float64) * h
        if jitter != 0.0:
            u = uniform01(seed, node_ids * 3 + axis)
            d = (2.0 * u - 1.0) * (jitter * h)
            movable = (idx > 0) & (idx < n)
            c = np.where(movable, c + d, c)
        coords.append(c)
    x, y, z = coords
    if bump is not None:
        height, width, x0 = bump
        zb = np.array([height * math.exp(-((xv - x0) / width) ** 2) for xv in x.tolist()],
                      dtype=np.float64)
        zeta = z / lz
        z = zb + (lz - zb) * zeta

    return x, y, z


def box_mesh(nx: int, ny: int, nz: int, lx: float = 1.0, ly: float = 1.0,
             lz: float = 1.0, jitter: float = 0.15, seed: int = 1,
             bc_types=(FAR_FIELD,) * 6, bump=None) -> RawMesh:
    """Kuhn-split hex block on ``[0,lx]x[0,ly]x[0,lz]``.

    ``jitter`` is the half-width, in units of the local spacing, of the
    uniform displacement applied to every coordinate that does not lie on a
    boundary plane (boundary nodes stay on their planes).  ``bc_types`` gives
    the BC type of the patches x-, x+, y-, y+, z-, z+ (patch ids 1..6).
    ``bump=(height, width, x0)`` lifts the bottom wall to
    ``zb(x) = height*exp(-((x-x0)/width)^2)`` and stretches each column as
    ``z = zb + (lz - zb) * zeta``.
    """
    nx, ny, nz = int(nx), int(ny), int(nz)
    x, y, z = _box_nodes(nx, ny, nz, lx, ly, lz, jitter, seed, bump)
    nhex = nx * ny * nz
    hidx = np.arange(nhex, dtype=np.int64)
    hi = hidx % nx
    hj = (hidx // nx) % ny
    hk = hidx // (nx * ny)
    hijk = (hi, hj, hk)
    nmax = (nx, ny, nz)

    def corner(p, steps):
        """Node ids of hex corners reached by unit steps along ``steps`` axes."""
        off = [hi.copy(), hj.copy(), hk.copy()]
        for ax in steps:
            off[ax] = off[ax] + 1
        return _node_id(off[0], off[1], off[2], nx, ny)

    # tet vertices per permutation
    tverts = []
    for (a, b, c) in PERMS:
        tverts.append((corner(None, ()), corner(None, (a,)), corner(None, (a, b)),
                       corner(None, (a, b, c))))

    faces_a = []   # cell A
    faces_b = []   # cell B (>=0) or -patch
    faces_n = []   # three node ids (unoriented)
    slot_keys = []  # boundary ordering key: local slot of the face in cell A

    # intra-hex faces: pi ~ s12(pi) share face opposite v1; pi ~ s23(pi) opposite v2
    for p, (a, b, c) in enumerate(PERMS):
        v0, v1, v2, v3 = tverts[p]
        q12 = _PERM_INDEX[(b, a, c)]
        if p < q12:
            faces_a.append(6 * hidx + p)
            faces_b.append(6 * hidx + q12)
            faces_n.append(np.stack([v0, v2, v3], axis=1))
            slot_keys.append(np.full(nhex, 1, dtype=np.int64))
        q23 = _PERM_INDEX[(a, c, b)]
        if p < q23:
            faces_a.append(6 * hidx + p)
            faces_b.append(6 * hidx + q23)
            faces_n.append(np.stack([v0, v1, v3], axis=1))
            slot_keys.append(np.full(nhex, 2, dtype=np.int64))
    # +a faces (opposite v0) : neighbour hex +e_a, perm (b, c, a); boundary at the top
    # -c faces (opposite v3) : emitted only on the boundary (interior ones come from +a)
    for p, (a, b, c) in enumerate(PERMS):
        v0, v1, v2, v3 = tverts[p]
        top = hijk[a] == nmax[a] - 1
        nb_hex = hidx + np.array([1, nx, nx * ny])[a]
        nb_cell = 6 * nb_hex + _PERM_INDEX[(b, c, a)]
        patch_top = 2 * a + 2          # x+ = 2, y+ = 4, z+ = 6
        faces_a.append(6 * hidx + p)
        faces_b.append(np.where(top, -patch_top, nb_cell))
        faces_n.append(np.stack([v1, v2, v3], axis=1))
        slot_keys.append(np.full(nhex, 0, dtype=np.int64))
        bot = hijk[c] == 0
        patch_bot = 2 * c + 1          # x- = 1, y- = 3, z- = 5
        sel = np.nonzero(bot)[0]
        faces_a.append(6 * hidx[sel] + p)
        faces_b.append(np.full(sel.shape[0], -patch_bot, dtype=np.int64))
        faces_n.append(np.stack([v0[sel], v1[sel], v2[sel]], axis=1))
        slot_keys.append(np.full(sel.shape[0], 3, dtype=np.int64))

    fa = np.concatenate(faces_a)
    fb = np.concatenate(faces_b)
    fn = np.concatenate(faces_n)
    fslot = np.concatenate(slot_keys)
    del faces_a, faces_b, faces_n, slot_keys

    is_b = fb < 0
    # c1 = lower cell for interior faces, the cell itself for boundary faces
    c1 = np.where(is_b, fa, np.minimum(fa, np.maximum(fb, 0)))
    c2 = np.where(is_b, fb, np.maximum(fa, fb))
    nb = int(is_b.sum())
    ncell = 6 * nhex
    # order: boundary faces by (c1, slot), then interior by (c1, c2)
    key_b = np.where(is_b, 0, 1).astype(np.int64)
    second = np.where(is_b, fslot, c2)
    order = np.lexsort((second, c1, key_b))
    c1 = c1[order]
    c2 = c2[order]
    fn = fn[order]
    del fa, fb, fslot, is_b, second, key_b, order

    # orient each face so that its normal points out of c1
    cv = np.stack([np.stack(tv, axis=1) for tv in tverts], axis=1)  # [nhex, 6, 4]
    cells_nodes = cv.reshape(ncell, 4)
    xyz = np.stack([x, y, z], axis=1)
    cc = xyz[cells_nodes].mean(axis=1)           # orientation test only
    p0 = xyz[fn[:, 0]]
    p1 = xyz[fn[:, 1]]
    p2 = xyz[fn[:, 2]]
    nrm = np.cross(p1 - p0, p2 - p0)
    fcen = (p0 + p1 + p2) / 3.0
    s = np.einsum("ij,ij->i", nrm, fcen - cc[c1])
    flip = s < 0.0
    fn[flip, 1], fn[flip, 2] = fn[flip, 2].copy(), fn[flip, 1].copy()

    f2c = np.empty(2 * c1.shape[0], dtype=np.int32)
    f2c[0::2] = c1
    f2c[1::2] = c2
    patches = [(pid, int(bc_types[pid - 1])) for pid in range(1, 7)]
    return RawMesh(x=np.ascontiguousarray(x), y=np.ascontiguousarray(y),
                   z=np.ascontiguousarray(z),
                   nnpf=np.full(c1.shape[0], 3, dtype=np.int32),
                   f2n=np.ascontiguousarray(fn.reshape(-1).astype(np.int32)),
                   f2c=f2c, n_cell=ncell, n_bface=nb, patches=patches)


def poly_mesh(x, y, z, cells, n_patch_types) -> RawMesh:
    """A FlowStar mesh from polyhedral cells.

    ``cells[c]`` lists the faces of cell ``c`` as ``(nodes, patch)``: the
    face's node ids in cyclic order and, for a face on the domain boundary,
    its patch id (1-based; None inside).  A face shared by two cells appears
    once in each.  Faces come out in the layout ``box_mesh`` documents:
    boundary faces first by (cell, local slot), interior faces by (lower
    cell, higher cell) with ``c1`` the lower cell, each face's nodes ordered
    so that its normal (Newell's, about the node mean) points out of ``c1``
    (the cyclic order reversed behind the first node otherwise).
    ``n_patch_types`` gives the BC type of patches 1, 2, ...
    """
    x = np.asarray(x, np.float64)
    y = np.asarray(y, np.float64)
    z = np.asarray(z, np.float64)
    open_faces = {}
    interior = []   # (c1, c2, nodes of the c1 side)
    boundary = []   # (c, slot, nodes, patch)
    for c, flist in enumerate(cells):
        for slot, (nodes, patch) in enumerate(flist):
            key = tuple(sorted(nodes))
            other = open_faces.pop(key, None)
            if other is None:
                open_faces[key] = (c, slot, tuple(nodes), patch)
            else:
                oc, _, onodes, _ = other
                c1, c2 = (oc, c) if oc < c else (c, oc)
                interior.append((c1, c2, onodes if oc < c else tuple(nodes)))
    for key, (c, slot, nodes, patch) in open_faces.items():
        if patch is None:
            raise ValueError(f"face {nodes} of cell {c} has no neighbour and no patch")
        boundary.append((c, slot, nodes, patch))
    boundary.sort(key=lambda t: (t[0], t[1]))
    interior.sort(key=lambda t: (t[0], t[1]))
    ncell = len(cells)
    cnodes = [sorted({n for nodes, _ in flist for n in nodes}) for flist in cells]
    cc = np.array([[x[v].mean(), y[v].mean(), z[v].mean()] for v in cnodes])

    def oriented(nodes, c1):
        v = np.array(nodes)
        px, py, pz = x[v], y[v], z[v]
        qx, qy, qz = np.roll(px, -1), np.roll(py, -1), np.roll(pz, -1)
        nrm = np.array([np.sum((py - qy) * (pz + qz)), np.sum((pz - qz) * (px + qx)),
                        np.sum((px - qx) * (py + qy))])
        fc = np.array([px.mean(), py.mean(), pz.mean()])
        if float(np.dot(nrm, fc - cc[c1])) < 0.0:
            nodes = (nodes[0],) + tuple(reversed(nodes[1:]))
        return nodes

    f2n, nnpf, f2c = [], [], []
    for c, _, nodes, patch in boundary:
        nodes = oriented(nodes, c)
        f2n.extend(nodes)
        nnpf.append(len(nodes))
        f2c.extend((c, -patch))
    for c1, c2, nodes in interior:
        nodes = oriented(nodes, c1)
        f2n.extend(nodes)
        nnpf.append(len(nodes))
        f2c.extend((c1, c2))
    patches = [(pid, int(t)) for pid, t in enumerate(n_patch_types, start=1)]
    return RawMesh(x=np.ascontiguousarray(x), y=np.ascontiguousarray(y),
                   z=np.ascontiguousarray(z), nnpf=np.array(nnpf, np.int32),
                   f2n=np.array(f2n, np.int32), f2c=np.array(f2c, np.int32), n_cell=ncell,
                   n_bface=len(boundary), patches=patches)


def hexprism_mesh(nx: int, ny: int, nz: int, jitter: float = 0.1, seed: int = 1,
                  bc_types=(FAR_FIELD,) * 6, prism_columns=lambda i, j: (i + j) % 2 == 0,
                  bump=None) -> RawMesh:
    """A mixed hexahedron / triangular-prism block on the unit cube: the hex
    columns (i, j) for which ``prism_columns`` holds are split by their
    vertical diagonal plane into two prisms per layer (the split is
    conforming: prisms meet prisms on triangles, hexes on whole quads).
    Nodes, jitter, bump and patches (x-, x+, y-, y+, z-, z+ = 1..6) as in
    ``box_mesh``; cells in hex order ``i + nx*(j + ny*k)``, a split hex
    giving two consecutive cells."""
    nx, ny, nz = int(nx), int(ny), int(nz)
    x, y, z = _box_nodes(nx, ny, nz, 1.0, 1.0, 1.0, jitter, seed, bump)

    def nid(i, j, k):
        return i + (nx + 1) * (j + (ny + 1) * k)

    cells = []
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                v = {(a, b, c): nid(i + a, j + b, k + c)
                     for a in (0, 1) for b in (0, 1) for c in (0, 1)}
                q = lambda *corners: tuple(v[t] for t in corners)  # noqa: E731
                xm = (q((0, 0, 0), (0, 0, 1), (0, 1, 1), (0, 1, 0)), 1 if i == 0 else None)
                xp = (q((1, 0, 0), (1, 1, 0), (1, 1, 1), (1, 0, 1)), 2 if i == nx - 1 else None)
                ym = (q((0, 0, 0), (1, 0, 0), (1, 0, 1), (0, 0, 1)), 3 if j == 0 else None)
                yp = (q((0, 1, 0), (0, 1, 1), (1, 1, 1), (1, 1, 0)), 4 if j == ny - 1 else None)
                bot, top = (5 if k == 0 else None), (6 if k == nz - 1 else None)
                if not prism_columns(i, j):
                    cells.append([xm, xp, ym, yp,
                                  (q((0, 0, 0), (0, 1, 0), (1, 1, 0), (1, 0, 0)), bot),
                                  (q((0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)), top)])
                    continue
                diag = (q((0, 0, 0), (1, 1, 0), (1, 1, 1), (0, 0, 1)), None)
                cells.append([ym, xp, diag,
                              (q((0, 0, 0), (1, 1, 0), (1, 0, 0)), bot),
                              (q((0, 0, 1), (1, 0, 1), (1, 1, 1)), top)])
                cells.append([xm, yp, diag,
                              (q((0, 0, 0), (0, 1, 0), (1, 1, 0)), bot),
                              (q((0, 0, 1), (1, 1, 1), (0, 1, 1)), top)])
    return poly_mesh(x, y, z, cells, bc_types)


def merged_hex_mesh(nx: int, ny: int, nz: int, jitter: float = 0.1, seed: int = 1,
                    bc_types=(FAR_FIELD,) * 6, merge=lambda i, j, k: (j + k) % 2 == 0,
                    at_boundary: bool = False, bump=None) -> RawMesh:
    """A hex block (``nx`` even) in which the hex pairs (i, i+1) with even i
    and ``merge(i, j, k)`` form one cell of 10 faces and 12 nodes (the pair's
    shared face removed): an interior merged cell has 5 neighbours before it
    and 5 after it in the cell order.  Pairs on the boundary merge only with
    ``at_boundary`` (they then have up to 10 faces after them, ghosts
    included).  Nodes and patches as in ``box_mesh``."""
    nx, ny, nz = int(nx), int(ny), int(nz)
    if nx % 2:
        raise ValueError("nx must be even")
    x, y, z = _box_nodes(nx, ny, nz, 1.0, 1.0, 1.0, jitter, seed, bump)

    def nid(i, j, k):
        return i + (nx + 1) * (j + (ny + 1) * k)

    def hex_faces(i, j, k):
        v = {(a, b, c): nid(i + a, j + b, k + c) for a in (0, 1) for b in (0, 1) for c in (0, 1)}
        q = lambda *corners: tuple(v[t] for t in corners)  # noqa: E731
        return {"xm": (q((0, 0, 0), (0, 0, 1), (0, 1, 1), (0, 1, 0)), 1 if i == 0 else None),
                "xp": (q((1, 0, 0), (1, 1, 0), (1, 1, 1), (1, 0, 1)), 2 if i == nx - 1 else None),
                "ym": (q((0, 0, 0), (1, 0, 0), (1, 0, 1), (0, 0, 1)), 3 if j == 0 else None),
                "yp": (q((0, 1, 0), (0, 1, 1), (1, 1, 1), (1, 1, 0)), 4 if j == ny - 1 else None),
                "zm": (q((0, 0, 0), (0, 1, 0), (1, 1, 0), (1, 0, 0)), 5 if k == 0 else None),
                "zp": (q((0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)), 6 if k == nz - 1 else None)}

    order = ("xm", "xp", "ym", "yp", "zm", "zp")
    cells = []
    for k in range(nz):
        for j in range(ny):
            for i in range(0, nx, 2):
                a, b = hex_faces(i, j, k), hex_faces(i + 1, j, k)
                inner = 0 < i and i + 2 < nx and 0 < j < ny - 1 and 0 < k < nz - 1
                if merge(i, j, k) and (inner or at_boundary):
                    cells.append([a["xm"], b["xp"], a["ym"], b["ym"], a["yp"], b["yp"],
                                  a["zm"], b["zm"], a["zp"], b["zp"]])
                else:
                    cells.append([a[f] for f in order])
                    cells.append([b[f] for f in order])
    return poly_mesh(x, y, z, cells, bc_types)


def cube_mesh(n: int, jitter: float = 0.15, seed: int = 1) -> RawMesh:
    """Unit cube, ``n^3`` hexes x 6 tets, far-field on every side."""
    return box_mesh(n, n, n, jitter=jitter, seed=seed)


def channel_mesh(nx: int = 192, ny: int = 48, nz: int = 48, jitter: float = 0.1,
                 seed: int = 5) -> RawMesh:
    """4x1x1 channel with a Gaussian bump on a slip wall at the bottom."""
    bc = (FAR_FIELD, FAR_FIELD, FAR_FIELD, FAR_FIELD, WALL, FAR_FIELD)
    return box_mesh(nx, ny, nz, lx=4.0, ly=1.0, lz=1.0, jitter=jitter, seed=seed,
                    bc_types=bc, bump=(0.05, 0.2, 1.5))


# ---------------------------------------------------------------------------
# FlowStar binary grid + bc.para text, as read by load_grid.cpp:129-314
# ---------------------------------------------------------------------------

def write_mfl(mesh: RawMesh, path: str) -> None:
    """Write the binary grid layout read by ``ReadMFlowGrid_binary``.

    The reader only stops before its interface block when ``feof`` is
    already set (load_grid.cpp:235), which it never is after an exact read,
    so a serial file ends with ``nIFace = 0`` and ``nINode = 0``.
    """
    with open(path, "wb") as f:
        np.array([mesh.n_node, mesh.n_face, mesh.n_cell], dtype=np.int32).tofile(f)
        mesh.x.astype(np.float64).tofile(f)
        mesh.y.astype(np.float64).tofile(f)
        mesh.z.astype(np.float64).tofile(f)
        mesh.nnpf.astype(np.int32).tofile(f)
        mesh.f2n.astype(np.int32).tofile(f)
        mesh.f2c.astype(np.int32).tofile(f)
        np.array([0, 0], dtype=np.int32).tofile(f)


def read_mfl(path: str) -> RawMesh:
    """Read a serial FlowStar binary grid; flips boundary faces the way the
    reference does (load_grid.cpp:209-229) and counts ``nBFace``."""
    with open(path, "rb") as f:
        buf = f.read()
    off = 0

    def take(dtype, count):
        nonlocal off
        arr = np.frombuffer(buf, dtype=dtype, count=count, offset=off)
        off += arr.nbytes
        return arr.copy()

    n_node, n_face, n_cell = (int(v) for v in take(np.int32, 3))
    x = take(np.float64, n_node)
    y = take(np.float64, n_node)
    z = take(np.float64, n_node)
    nnpf = take(np.int32, n_face)
    f2n = take(np.int32, int(nnpf.sum()))
    f2c = take(np.int32, 2 * n_face)
    ptr = np.concatenate([[0], np.cumsum(nnpf)])
    nb = 0
    for i in range(n_face):
        if f2c[2 * i] < 0:
            s, e = ptr[i] + 1, ptr[i + 1]
            f2n[s:e] = f2n[s:e][::-1].copy()
            f2c[2 * i], f2c[2 * i + 1] = f2c[2 * i + 1], f2c[2 * i]
            nb += 1
        elif f2c[2 * i + 1] < 0:
            nb += 1
    return RawMesh(x=x, y=y, z=z, nnpf=nnpf, f2n=f2n, f2c=f2c, n_cell=n_cell,
                   n_bface=nb, patches=[])


def write_bc(mesh: RawMesh, path: str) -> None:
    """``bc.para``: patch count, then ``patch_id type`` lines
    (``ReadMFlowBoundaryCondition``, load_grid.cpp:282-314)."""
    with open(path, "w") as f:
        f.write(f"{len(mesh.patches)}\n")
        for pid, typ in mesh.patches:
            f.write(f"{pid} {typ}\n")


def bface_types(mesh: RawMesh) -> np.ndarray:
    """BC type of each boundary face, as ``SpecifyBC`` assigns it
    (load_grid.cpp:893-901: record ``-c2 - 1`` of the bc table)."""
    table = {pid: typ for pid, typ in mesh.patches}
    ids = -mesh.f2c[1:2 * mesh.n_bface:2]
    ordered = [typ for _, typ in mesh.patches]
    return np.array([ordered[i - 1] for i in ids.tolist()], dtype=np.int32) \
        if len(table) else np.zeros(mesh.n_bface, dtype=np.int32)
