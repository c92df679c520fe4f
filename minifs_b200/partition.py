"""One mesh split into parts, each iterated by its own context (one per GPU):
the counterpart of the reference's MPI mode (src/Base/parallel_mpi.cpp,
PassInterfaceData in src/Kernels/load_grid.cpp:912-942) for the iteration
path.

Each part is an ordinary FlowStar mesh of its cells.  A face between two
parts becomes, in each of them, a boundary face of type INTERFACE (10) whose
ghost holds the other part's cell -- the reference's own representation of a
partition cut (its ghost update skips the type, load_grid.cpp:1030-1031; the
gradient takes node means there, cal_gradient.cpp:1749) -- and the part
carries the FlowStar interface block that names, for every such face and
every node shared with another part, the zone and the index on the other
side (the block ``flowstar.write_grid`` stores).

``split`` makes the parts, ``halo_lists`` turns one part's interface block
into the exchange lists of ``mfg_halo_set``, ``prepare_parts`` runs the
preprocessing per part with the node data of the whole mesh, and
``Decomposed`` iterates the parts in step through ``mfg_halo_phase`` with
the exchanges in between, either all parts in this process (``LocalExchange``,
device copies) or one part per rank (``DistExchange``, torch.distributed:
NCCL on GPUs).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .flowstar import Interfaces
from .meshgen import INTERFACE, RawMesh


@dataclass
class Part:
    mesh: RawMesh            # the part as a FlowStar mesh (its patches plus the interface patch)
    interfaces: Interfaces   # FlowStar interface block, zones numbered from 0
    rank: int                # zone of this part
    cells: np.ndarray        # whole-mesh cell of each local cell (ascending)
    nodes: np.ndarray        # whole-mesh node of each local node (ascending)
    bfaces: np.ndarray       # whole-mesh boundary face of each of the part's own boundary faces
    iface_cells: np.ndarray  # whole-mesh cell on the other side of each interface face
    n_own_bface: int = 0     # boundary faces before the interface faces


def slab_parts(n_cell: int, world: int) -> np.ndarray:
    """Part of every cell: `world` contiguous, balanced ranges of the cell
    numbering (slabs of hex layers on the generated block meshes)."""
    if world < 1:
        raise ValueError("at least one part")
    return (np.arange(n_cell, dtype=np.int64) * world // max(n_cell, 1)).astype(np.int32)


def cell_points(mesh: RawMesh) -> np.ndarray:
    """A point inside every cell: the mean of its faces' node means [C][3]."""
    nnpf = np.asarray(mesh.nnpf, np.int64)
    fptr = np.concatenate([[0], np.cumsum(nnpf)])
    f2n = np.asarray(mesh.f2n, np.int64)
    xyz = np.stack([np.asarray(mesh.x), np.asarray(mesh.y), np.asarray(mesh.z)], 1)
    fsum = np.add.reduceat(xyz[f2n], fptr[:-1], axis=0) if f2n.size else np.zeros((0, 3))
    fmean = fsum / np.maximum(nnpf, 1)[:, None]
    f2c = np.asarray(mesh.f2c, np.int64).reshape(-1, 2)
    acc = np.zeros((mesh.n_cell, 3))
    cnt = np.zeros(mesh.n_cell)
    for side in (0, 1):
        c = f2c[:, side]
        ok = c >= 0
        np.add.at(acc, c[ok], fmean[ok])
        np.add.at(cnt, c[ok], 1.0)
    return acc / np.maximum(cnt, 1.0)[:, None]


def rcb_parts(mesh: RawMesh, world: int) -> np.ndarray:
    """Part of every cell by recursive coordinate bisection of the cells'
    points: each step cuts the longest extent so that the two sides get
    cells in proportion to the parts they will hold."""
    if world < 1:
        raise ValueError("at least one part")
    pts = cell_points(mesh)
    part_of = np.zeros(mesh.n_cell, np.int32)

    def cut(idx, first, count):
        if count == 1 or idx.size == 0:
            part_of[idx] = first
            return
        left = count // 2
        ext = pts[idx].max(0) - pts[idx].min(0)
        axis = int(np.argmax(ext))
        order = idx[np.argsort(pts[idx, axis], kind="stable")]
        k = (order.size * left) // count
        cut(order[:k], first, left)
        cut(order[k:], first + left, count - left)

    cut(np.arange(mesh.n_cell), 0, world)
    return part_of


def split(mesh: RawMesh, part_of, world: int) -> list[Part]:
    """The parts of `mesh` for the cell -> part map `part_of` (values in
    [0, world)).

    Local cells and nodes keep the whole mesh's order.  Faces of a part: its
    own boundary faces, then its interface faces, then its interior faces,
    each group in the whole mesh's order.  An interface face whose inner cell
    is the face's second cell is turned round as the reference's reader turns
    a face with a boundary on its left (load_grid.cpp:214-221): first node
    kept, the others reversed, so that its normal points out of the part.
    """
    part_of = np.asarray(part_of, np.int32)
    if part_of.shape != (mesh.n_cell,):
        raise ValueError("part_of needs one entry per cell")
    if world < 1 or part_of.min(initial=0) < 0 or part_of.max(initial=0) >= world:
        raise ValueError("part numbers must lie in [0, world)")
    if np.any(np.bincount(part_of, minlength=world) == 0):
        raise ValueError("every part needs at least one cell")
    f2c = np.asarray(mesh.f2c, np.int64).reshape(-1, 2)
    nnpf = np.asarray(mesh.nnpf, np.int64)
    fptr = np.concatenate([[0], np.cumsum(nnpf)])
    f2n = np.asarray(mesh.f2n, np.int64)
    F, G = mesh.n_face, mesh.n_bface
    iface_patch = max([pid for pid, _ in mesh.patches] + [0]) + 1
    c1, c2 = f2c[:, 0], f2c[:, 1]
    p1 = part_of[c1]
    p2 = np.where(c2 >= 0, part_of[np.maximum(c2, 0)], -1)
    fidx = np.arange(F)
    interior = fidx >= G
    cut = interior & (p1 != p2)
    # each part's own boundary faces, cut faces and interior faces
    sides = []
    for p in range(world):
        own_b = fidx[(~interior) & (p1 == p)]
        cut_p = fidx[cut & ((p1 == p) | (p2 == p))]
        inner = fidx[interior & (p1 == p) & (p2 == p)]
        sides.append((own_b, cut_p, inner))
    # local boundary-face index of each cut face in each of its two parts
    cut_local = np.full((world, F), -1, np.int64)
    for p, (own_b, cut_p, _) in enumerate(sides):
        cut_local[p, cut_p] = own_b.size + np.arange(cut_p.size)
    parts = []
    for p, (own_b, cut_p, inner) in enumerate(sides):
        cells = np.nonzero(part_of == p)[0]
        local = np.full(mesh.n_cell, -1, np.int64)
        local[cells] = np.arange(cells.size)
        faces = np.concatenate([own_b, cut_p, inner])
        turned = np.zeros(faces.size, bool)
        ncut = cut_p.size
        cs = slice(own_b.size, own_b.size + ncut)
        turned[cs] = p1[cut_p] != p  # inner cell on the right: turned round
        inner_c = np.where(turned[cs], c2[cut_p], c1[cut_p])
        outer_c = np.where(turned[cs], c1[cut_p], c2[cut_p])
        lf2c = np.empty((faces.size, 2), np.int64)
        lf2c[:own_b.size, 0] = local[c1[own_b]]
        lf2c[:own_b.size, 1] = c2[own_b]
        lf2c[cs, 0] = local[inner_c]
        lf2c[cs, 1] = -iface_patch
        lf2c[own_b.size + ncut:, 0] = local[c1[inner]]
        lf2c[own_b.size + ncut:, 1] = local[c2[inner]]
        other = np.where(turned[cs], p1[cut_p], p2[cut_p])
        # node lists: each face's nodes, a turned face's after its first node
        # reversed
        cnt = nnpf[faces]
        start = fptr[faces]
        optr = np.concatenate([[0], np.cumsum(cnt)])
        pos = np.arange(optr[-1]) - np.repeat(optr[:-1], cnt)   # position within the face
        rev = np.where(pos == 0, 0, np.repeat(cnt, cnt) - pos)  # reversed position
        src = np.repeat(start, cnt) + np.where(np.repeat(turned, cnt), rev, pos)
        allnodes = f2n[src]
        used = np.unique(allnodes)
        nmap = np.full(mesh.n_node, -1, np.int64)
        nmap[used] = np.arange(used.size)
        raw = RawMesh(x=np.ascontiguousarray(mesh.x[used], np.float64),
                      y=np.ascontiguousarray(mesh.y[used], np.float64),
                      z=np.ascontiguousarray(mesh.z[used], np.float64),
                      nnpf=cnt.astype(np.int32),
                      f2n=nmap[allnodes].astype(np.int32),
                      f2c=lf2c.reshape(-1).astype(np.int32),
                      n_cell=int(cells.size), n_bface=int(own_b.size + ncut),
                      patches=list(mesh.patches) + [(iface_patch, INTERFACE)])
        parts.append(Part(mesh=raw,
                          interfaces=Interfaces(nbz=other.astype(np.int32),
                                                nbf=cut_local[other, cut_p].astype(np.int32)),
                          rank=p, cells=cells.astype(np.int32), nodes=used.astype(np.int32),
                          bfaces=own_b.astype(np.int32), iface_cells=outer_c.astype(np.int32),
                          n_own_bface=int(own_b.size)))
    # the node half of the interface block: every node shared with another
    # part, once per such part, with its index there, ordered by (zone,
    # own index, index there)
    zone = np.concatenate([np.full(pt.nodes.size, pt.rank, np.int64) for pt in parts])
    lidx = np.concatenate([np.arange(pt.nodes.size, dtype=np.int64) for pt in parts])
    glob = np.concatenate([pt.nodes.astype(np.int64) for pt in parts])
    order = np.lexsort((zone, glob))  # by node, then zone
    glob, zone, lidx = glob[order], zone[order], lidx[order]
    first = np.concatenate([[0], np.nonzero(np.diff(glob))[0] + 1])
    mult = np.diff(np.concatenate([first, [glob.size]]))
    ent = [[] for _ in range(world)]
    for f0, m in zip(first[mult > 1].tolist(), mult[mult > 1].tolist()):
        zs, ls = zone[f0:f0 + m].tolist(), lidx[f0:f0 + m].tolist()
        for a_ in range(m):
            for b_ in range(m):
                if a_ != b_:
                    ent[zs[a_]].append((zs[b_], ls[a_], ls[b_]))
    for pt in parts:
        e = np.array(sorted(ent[pt.rank]), np.int64).reshape(-1, 3)
        pt.interfaces.nbsn = e[:, 1].astype(np.int32)
        pt.interfaces.nbzn = e[:, 0].astype(np.int32)
        pt.interfaces.nbrn = e[:, 2].astype(np.int32)
    return parts


@dataclass
class HaloLists:
    """Exchange lists of one part (the arguments of mfg_halo_set), one
    segment per neighbour, neighbours ascending.  Within the segments shared
    by zones p < r, faces and nodes are ordered by their index in p, so that
    the rows p sends are the rows r expects and the reverse."""
    rank: int
    neighbors: list = field(default_factory=list)
    send_cells: np.ndarray = None   # local cell of each sent row
    recv_bfaces: np.ndarray = None  # local interface face whose ghost each received row fills
    nodes: np.ndarray = None        # local node of each node entry
    row_ptr: np.ndarray = None      # segment bounds of the rows (sent and received alike)
    node_ptr: np.ndarray = None     # segment bounds of the node entries


def halo_lists(mesh: RawMesh, interfaces: Interfaces, rank: int) -> HaloLists:
    """The exchange lists of zone `rank` from its own mesh and interface
    block alone (what one process reading its own grid file has)."""
    itf = interfaces
    G = mesh.n_bface
    f2c = np.asarray(mesh.f2c, np.int64).reshape(-1, 2)
    nif = len(itf.nbz)
    ib = np.arange(G - nif, G, dtype=np.int64)  # interface faces close the boundary block
    if nif and np.any(f2c[ib, 1] >= 0):
        raise ValueError("interface faces must be the last boundary faces")
    nbz, nbf = np.asarray(itf.nbz, np.int64), np.asarray(itf.nbf, np.int64)
    nbzn = np.asarray(itf.nbzn, np.int64)
    nbsn, nbrn = np.asarray(itf.nbsn, np.int64), np.asarray(itf.nbrn, np.int64)
    neighbors = sorted(set(nbz.tolist()) | set(nbzn.tolist()))
    send, recv, nodes, row_ptr, node_ptr = [], [], [], [0], [0]
    for r in neighbors:
        sel = np.nonzero(nbz == r)[0]
        key = ib[sel] if rank < r else nbf[sel]
        sel = sel[np.argsort(key, kind="stable")]
        recv.append(ib[sel])
        send.append(f2c[ib[sel], 0])
        row_ptr.append(row_ptr[-1] + sel.size)
        seln = np.nonzero(nbzn == r)[0]
        keyn = nbsn[seln] if rank < r else nbrn[seln]
        seln = seln[np.argsort(keyn, kind="stable")]
        nodes.append(nbsn[seln])
        node_ptr.append(node_ptr[-1] + seln.size)

    def cat(v):
        return np.concatenate(v).astype(np.int32) if v else np.zeros(0, np.int32)

    return HaloLists(rank=rank, neighbors=neighbors, send_cells=cat(send), recv_bfaces=cat(recv),
                     nodes=cat(nodes), row_ptr=np.array(row_ptr, np.int64),
                     node_ptr=np.array(node_ptr, np.int64))


def prepare_parts(mesh: RawMesh, params, parts: list[Part], bump_amp: float = 0.05,
                  bump_sigma: float = 0.1, bump_center=(0.5, 0.5, 0.5)):
    """Preprocessing of every part (``grid.prepare``) with the node data of
    the whole mesh: node weights, marks and symmetry normals are sums and
    minima over the parts in the reference (CommInternodeDataMPI /
    CommInternodeDataMPI2, grid_polyhedra_auxiliary_functions.cpp:951-1047,
    :2114-2119), here taken from the whole mesh's preprocessing; the
    initial state is the whole mesh's, each interface ghost holding the
    neighbouring cell (PassInterfaceData after AllocAndInitFlowfield,
    load_grid.cpp:505-507).  Returns (whole-mesh grid, part grids)."""
    from . import grid as gr
    kw = dict(bump_amp=bump_amp, bump_sigma=bump_sigma, bump_center=bump_center)
    whole = gr.prepare(mesh, params, **kw)
    C = whole.n_cell
    q = whole.q0.reshape(5, whole.n)
    out = []
    for pt in parts:
        pg = gr.prepare(pt.mesh, params, **kw)
        for k in ("wnode", "nmark", "nodesymm", "xfn_n_symm", "yfn_n_symm", "zfn_n_symm"):
            pg.arrays[k] = np.ascontiguousarray(whole.arrays[k][pt.nodes])
        rows = np.concatenate([pt.cells, C + pt.bfaces.astype(np.int64), pt.iface_cells])
        pg.q0 = np.ascontiguousarray(q[:, rows].reshape(-1))
        out.append(pg)
    return whole, out


# kinds of the node-weight passes of ComputeWeight3D_Node
# (grid_polyhedra_auxiliary_functions.cpp:929-1001): wall faces, far-field
# faces (both far-field types), then the other types bar symmetry and
# interfaces; the mark each gives a node
_KIND_MARK = {1: 3, 2: 6, 3: 101}


def _face_kinds(bctype) -> np.ndarray:
    t = np.asarray(bctype, np.int64)
    kind = np.zeros(t.size, np.int64)
    kind[t == 3] = 1
    kind[(t == 6) | (t == 61)] = 2
    kind[~np.isin(t, (3, 4, 6, 61, 10))] = 3
    return kind


def _add_received(local: np.ndarray, lists: HaloLists, recv: np.ndarray, combine) -> np.ndarray:
    """A node's own value combined with every neighbour's entry for it, the
    entries in order (RecvSendVarNeighbor_Node, parallel_mpi.cpp:1997-2004)."""
    out = local.copy()
    for e, nd in enumerate(lists.nodes.tolist()):
        out[nd] = combine(out[nd], recv[e])
    return out


def zone_node_data(pgs: dict, lists: dict, exchange, device="cpu") -> None:
    """The node data of zones that know only their own grids: node marks,
    weights and symmetry normals combined over the zones as the reference's
    MPI build does at set-up (CommInternodeDataMPI2 / CommInternodeDataMPI,
    grid_polyhedra_auxiliary_functions.cpp:951-1047 and :2114-2119).
    `pgs` maps zone -> its PreparedGrid (from ``grid.prepare`` of its own
    mesh; its wnode, nmark, nodesymm and symmetry normals are replaced),
    `lists` zone -> HaloLists; `exchange` moves the node entries between
    the zones (``LocalExchange`` or ``DistExchange``; every process calls
    this with its own zones)."""
    import torch
    bufs = {z: HaloBuffers(lists[z], device) for z in pgs}

    def swap(values):
        for z, b in bufs.items():
            v = np.zeros((max(lists[z].nodes.size, 1), 8))
            v[:lists[z].nodes.size, :values[z].shape[1]] = values[z]
            b.node_send.copy_(torch.from_numpy(v))
        exchange.nodes(bufs)
        return {z: b.node_recv.cpu().numpy()[:lists[z].nodes.size] for z, b in bufs.items()}

    geo = {}
    for z, pg in pgs.items():
        A = pg.arrays
        N, G = pg.n_node, pg.n_bface
        nnpf = np.asarray(A["nnpf"], np.int64)
        fptr = np.concatenate([[0], np.cumsum(nnpf)])
        f2n = np.asarray(A["f2n"], np.int64)
        kind = _face_kinds(A["bctype"][:G])
        # per boundary-face node: its face (faces and their nodes in order)
        bface = np.repeat(np.arange(G), nnpf[:G])
        bnode = f2n[:fptr[G]]
        has = np.zeros((N, 3))
        k = kind[bface]
        has[bnode[k > 0], k[k > 0] - 1] = 1.0
        sym = np.zeros((N, 5))  # flag, sums of the normals, face count
        s4 = np.asarray(A["bctype"][:G])[bface] == 4
        sym[bnode[s4], 0] = 1.0
        # np.add.at adds in index order: FindNodeSYMM's loop order
        for col, name in ((1, "xfn"), (2, "yfn"), (3, "zfn")):
            np.add.at(sym[:, col], bnode[s4], np.asarray(A[name])[bface[s4]])
        np.add.at(sym[:, 4], bnode[s4], 1.0)
        geo[z] = (fptr, f2n, kind, has, sym)
    recv = swap({z: np.concatenate([g[3], g[4]], 1)[lists[z].nodes] for z, g in geo.items()})
    marks = {}
    for z, pg in pgs.items():
        fptr, f2n, kind, has, sym = geo[z]
        both = np.concatenate([has, sym], 1)

        def comb(a, b):
            r = a + b
            r[:4] = np.maximum(a[:4], b[:4])  # flags: set on any zone
            return r

        both = _add_received(both, lists[z], recv[z], comb)
        hw, hf, ho = both[:, 0] > 0, both[:, 1] > 0, both[:, 2] > 0
        mark = np.where(hw, 3, np.where(hf, 6, np.where(ho, 101, 0))).astype(np.int32)
        marks[z] = mark
        sflag = both[:, 3] > 0
        A = pg.arrays
        A["nmark"] = mark
        A["nodesymm"] = sflag.astype(np.int32)
        for k, name in enumerate(("xfn_n_symm", "yfn_n_symm", "zfn_n_symm")):
            v = np.zeros(pg.n_node)
            v[sflag] = both[sflag, 4 + k] / both[sflag, 7]
            A[name] = v
    # each zone's share of the node weights under the combined marks, in the
    # passes' order (faces, then cells), then the sums over zones
    part = {}
    for z, pg in pgs.items():
        fptr, f2n, kind, has, sym = geo[z]
        A = pg.arrays
        mark = marks[z]
        w = np.zeros(pg.n_node)
        wb = np.asarray(A["wbface"])
        G = pg.n_bface
        bface = np.repeat(np.arange(G), np.diff(fptr[:G + 1]))
        bnode = f2n[:fptr[G]]
        # the passes' order: wall faces, far-field faces, the others, each in
        # face order; a node takes the faces of its mark's kind only
        for kd in (1, 2, 3):
            sel = (kind[bface] == kd) & (mark[bnode] == _KIND_MARK[kd])
            np.add.at(w, bnode[sel], wb[:fptr[G]][sel])
        c2n = np.asarray(A["c2n"], np.int64)
        wc = np.asarray(A["wc2n"])
        sel = mark[c2n] == 0
        np.add.at(w, c2n[sel], wc[sel])
        part[z] = w
    recv = swap({z: part[z][lists[z].nodes][:, None] for z in pgs})
    for z, pg in pgs.items():
        pg.arrays["wnode"] = _add_received(part[z], lists[z], recv[z][:, 0], lambda a, b: a + b)


def assemble(parts: list[Part], values: list[np.ndarray], n_cell: int, width: int = 5):
    """Whole-mesh cell array [width][n_cell] from per-part arrays laid out
    [width][n_local] (n_local = the part's cells, or cells + ghosts)."""
    out = np.zeros((width, n_cell))
    for pt, v in zip(parts, values):
        v = np.asarray(v).reshape(width, -1)
        out[:, pt.cells] = v[:, :pt.cells.size]
    return out


def build_zones(zones: dict, params, exchange=None, device_of=None, **bump) -> dict:
    """Contexts of zones known only from their own grids, as one process of
    the reference's MPI build reads its zone file: `zones` maps zone ->
    (mesh, interfaces), e.g. from ``flowstar.read_grid`` (the mesh's
    patches set from the zone's bc.para).  Each zone is preprocessed on its
    own, its node data combined with the other zones' through `exchange`
    (``zone_node_data``; every process passes its zones and the same
    exchange kind), and its context created on ``device_of(z)``; the
    interface ghosts get the neighbours' states in ``Decomposed``'s first
    exchange.  Returns {zone: HaloPart}."""
    import torch

    from . import grid as gr
    exchange = exchange if exchange is not None else LocalExchange()
    pgs, lists = {}, {}
    for z, (mesh, itf) in sorted(zones.items()):
        pgs[z] = gr.prepare(mesh, params, **bump)
        lists[z] = halo_lists(mesh, itf, z)
    dev0 = 0 if device_of is None else int(device_of(min(zones)))
    zone_node_data(pgs, lists, exchange,
                   device="cpu" if isinstance(exchange, LocalExchange) else
                   torch.device("cuda", dev0))
    streams, held = {}, {}
    for z in sorted(zones):
        dev = 0 if device_of is None else int(device_of(z))
        if dev not in streams:
            streams[dev] = torch.cuda.Stream(device=dev)
        held[z] = HaloPart(pgs[z], params, lists[z], streams[dev])
    return held


# ---- iteration -------------------------------------------------------------

class HaloBuffers:
    """The exchange buffers of one part (torch tensors on `device`): rows of
    8 doubles for cells and node entries, the dt extrema and the residual
    sums, laid out as ``mfg_halo`` describes."""

    def __init__(self, lists: HaloLists, device):
        import torch
        self.lists = lists
        self.device = torch.device(device)
        ns, nr, nn = lists.send_cells.size, lists.recv_bfaces.size, lists.nodes.size

        def buf(n):
            return torch.zeros((max(n, 1), 8), dtype=torch.float64, device=self.device)

        self.send_rows, self.recv_rows = buf(ns), buf(nr)
        self.node_send, self.node_recv = buf(nn), buf(nn)
        # second order: gradient, limiter and centroid rows of 24 doubles
        self.grad_send = torch.zeros((max(ns, 1), 24), dtype=torch.float64, device=self.device)
        self.grad_recv = torch.zeros((max(nr, 1), 24), dtype=torch.float64, device=self.device)
        self.ext = torch.zeros(2, dtype=torch.int64, device=self.device)
        self.norm_sq = torch.zeros(5, dtype=torch.float64, device=self.device)

    def seg(self, which: str, k: int):
        """Rows of segment k (the k-th neighbour) of a buffer."""
        ptr = self.lists.node_ptr if which.startswith("node") else self.lists.row_ptr
        return getattr(self, which)[int(ptr[k]):int(ptr[k + 1])]


class HaloPart(HaloBuffers):
    """One part's context with its exchange lists and buffers.  The context
    runs on `stream` (a torch.cuda.Stream of its device, shared by the parts
    on that device); the exchanges run on it too (``Decomposed`` makes it
    the current stream)."""

    def __init__(self, pg, params, lists: HaloLists, stream, precision: str = "fp64"):
        import ctypes as ct

        import torch

        from . import _lib
        from .solver import Solver
        self.stream = stream
        with torch.cuda.stream(stream):
            super().__init__(lists, stream.device)
        self.solver = Solver(pg, params, device=stream.device.index, precision=precision)
        h = _lib.Halo()
        keep = [np.ascontiguousarray(a, np.int32) for a in
                (lists.send_cells, lists.recv_bfaces, lists.nodes)]
        h.n_send, h.n_recv, h.n_node = (int(a.size) for a in keep)
        h.send_cells, h.recv_bfaces, h.nodes = (_lib.ptr(a, _lib.i32p) for a in keep)
        for name in ("send_rows", "recv_rows", "node_send", "node_recv", "ext", "norm_sq",
                     "grad_send", "grad_recv"):
            setattr(h, name, ct.c_void_p(getattr(self, name).data_ptr()))
        lib = self.solver.lib
        _lib.check("mfg_set_stream", lib.mfg_set_stream(self.solver.ctx,
                                                        ct.c_void_p(stream.cuda_stream)))
        _lib.check("mfg_halo_set", lib.mfg_halo_set(self.solver.ctx, ct.byref(h)))
        del keep

    def phase(self, ph: int, iter_done: int = 0):
        from . import _lib
        _lib.check("mfg_halo_phase", self.solver.lib.mfg_halo_phase(self.solver.ctx, int(ph),
                                                                      int(iter_done)))

    def close(self):
        self.solver.close()


def build_parts(mesh: RawMesh, params, world: int, part_of=None, zones=None, device_of=None,
                precision: str = "fp64", **bump) -> tuple:
    """Split `mesh` (slabs unless `part_of` is given), prepare every part and
    create the contexts of `zones` (default: all), zone z on CUDA device
    ``device_of(z)`` (default 0).  Returns (parts, whole-mesh grid,
    {zone: HaloPart})."""
    import torch
    if part_of is None:
        part_of = slab_parts(mesh.n_cell, world)
    parts = split(mesh, part_of, world)
    whole, pgs = prepare_parts(mesh, params, parts, **bump)
    zones = list(range(world)) if zones is None else list(zones)
    streams = {}
    held = {}
    for z in zones:
        dev = 0 if device_of is None else int(device_of(z))
        if dev not in streams:
            streams[dev] = torch.cuda.Stream(device=dev)
        pt = parts[z]
        held[z] = HaloPart(pgs[z], params, halo_lists(pt.mesh, pt.interfaces, z), streams[dev],
                           precision=precision)
    return parts, whole, held


class LocalExchange:
    """Every part in this process: exchanges as device copies (peer copies
    between GPUs), reductions on the device."""

    def rows(self, parts: dict):
        self._pairs(parts, "send_rows", "recv_rows")

    def nodes(self, parts: dict):
        self._pairs(parts, "node_send", "node_recv")

    def grads(self, parts: dict):
        self._pairs(parts, "grad_send", "grad_recv")

    @staticmethod
    def _pairs(parts, src, dst):
        for p, hp in parts.items():
            for k, r in enumerate(hp.lists.neighbors):
                other = parts[r]
                j = other.lists.neighbors.index(p)
                hp.seg(dst, k).copy_(other.seg(src, j), non_blocking=True)

    def extrema(self, parts: dict):
        import torch
        ranks = sorted(parts)
        ext = torch.stack([parts[r].ext.to(parts[ranks[0]].device) for r in ranks])
        g = torch.stack([ext[:, 0].max(), ext[:, 1].min()])
        for r in ranks:
            parts[r].ext.copy_(g, non_blocking=True)

    def sum(self, t):
        return t


class DistExchange:
    """One part (or several) per process, parts of other processes reached
    through torch.distributed point-to-point operations (NCCL over NVLink on
    GPUs); the reductions are all-reduces.  Each process must call every
    step in the same order."""

    def __init__(self, group=None):
        self.group = group

    def _p2p(self, parts, src, dst):
        import torch.distributed as dist
        ops = []
        local = set(parts)
        for p, hp in parts.items():
            for k, r in enumerate(hp.lists.neighbors):
                if r in local:
                    j = parts[r].lists.neighbors.index(p)
                    hp.seg(dst, k).copy_(parts[r].seg(src, j))
                    continue
                ops.append(dist.P2POp(dist.isend, hp.seg(src, k).contiguous(), r, self.group))
                ops.append(dist.P2POp(dist.irecv, hp.seg(dst, k), r, self.group))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()

    def rows(self, parts: dict):
        self._p2p(parts, "send_rows", "recv_rows")

    def nodes(self, parts: dict):
        self._p2p(parts, "node_send", "node_recv")

    def grads(self, parts: dict):
        self._p2p(parts, "grad_send", "grad_recv")

    def extrema(self, parts: dict):
        import torch
        import torch.distributed as dist
        LocalExchange().extrema(parts)
        hp = parts[min(parts)]
        mx, mn = hp.ext[0:1].clone(), hp.ext[1:2].clone()
        dist.all_reduce(mx, op=dist.ReduceOp.MAX, group=self.group)
        dist.all_reduce(mn, op=dist.ReduceOp.MIN, group=self.group)
        g = torch.cat([mx, mn])
        for p in parts.values():
            p.ext.copy_(g)

    def sum(self, t):
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)
        return t


class Decomposed:
    """Parts iterated in step: the main-loop body (main.cpp:201-291) with the
    reference's MPI exchanges (phases of ``mfg_halo_phase``).  ``parts``
    maps zone -> HaloPart for the zones this process holds."""

    def __init__(self, parts: dict, exchange=None):
        self.parts = dict(sorted(parts.items()))
        self.ex = exchange if exchange is not None else LocalExchange()
        self.iter_done = 0
        self.order = 1
        self.streams = []
        for hp in self.parts.values():
            if all(hp.stream is not s for s in self.streams):
                self.streams.append(hp.stream)
        for s in self.streams:
            s.synchronize()  # the buffers' allocation and zero fill
        with self._on_streams():
            self._initial_gradient()

    def _on_streams(self):
        import contextlib

        import torch
        stack = contextlib.ExitStack()
        for s in self.streams:
            stack.enter_context(torch.cuda.stream(s))
        return stack

    def _each(self, ph):
        for hp in self.parts.values():
            hp.phase(ph, self.iter_done)

    def _initial_gradient(self):
        """PassInterfaceData and the gradient of the initial state
        (load_grid.cpp:507, AllocAndCalQuantityGradient)."""
        from . import _lib
        self._each(_lib.HALO["pack_q"])
        self.ex.rows(self.parts)
        self._each(_lib.HALO["nodes"])
        self.ex.nodes(self.parts)
        self._each(_lib.HALO["gradient"])

    def set_order(self, order: int, venkat_k: float = 5.0):
        """The reference's `order` switch on every part (``mfg_set_order``):
        second order reconstructs the interface ghosts' face states from the
        neighbouring cells' gradients, limiters and centroids."""
        for hp in self.parts.values():
            hp.solver.set_order(order, venkat_k)
        self.order = int(order)

    def iterate(self, n: int) -> np.ndarray:
        """n iterations; returns the residual norms of every iteration over
        all parts, [n][5]."""
        import torch

        from . import _lib
        H = _lib.HALO
        first = next(iter(self.parts.values()))
        with self._on_streams():
            hist = torch.zeros((max(n, 1), 5), dtype=torch.float64, device=first.device)
            for i in range(n):
                if self.order >= 2:
                    self._each(H["limit"])
                    self.ex.grads(self.parts)
                self._each(H["face"])
                self.ex.extrema(self.parts)
                self._each(H["forward"])
                self.ex.rows(self.parts)
                self._each(H["backward"])
                self.ex.rows(self.parts)
                self._each(H["nodes"])
                self.ex.nodes(self.parts)
                self._each(H["gradient"])
                for hp in self.parts.values():
                    hist[i] += hp.norm_sq.to(first.device)
                self.iter_done += 1
            self._each(H["check"])
            hist = self.ex.sum(hist)
            out = torch.sqrt(hist[:n]).cpu().numpy()
        return out

    def download(self, field: str) -> dict:
        return {r: hp.solver.download(field) for r, hp in self.parts.items()}

    def close(self):
        for hp in self.parts.values():
            hp.close()
