"""Partitioned meshes on the CPU: the parts and their interface blocks, the
exchange lists built from one part's block alone, the per-part
preprocessing against the whole mesh's, the FlowStar round trip of a part,
and the exchanges themselves (in-process and as two gloo ranks) on host
buffers filled by a NumPy restatement of the packing."""
import os
import socket

import numpy as np
import pytest

from minifs_b200 import flowstar, grid as gr, meshgen
from minifs_b200 import partition as pa


def _mesh(kind="box"):
    if kind == "box":
        bc = (3, 6, 4, 61, 5, 6)
        m = meshgen.box_mesh(6, 5, 4, jitter=0.2, seed=3, bc_types=bc)
        m.patches = [(i + 1, t) for i, t in enumerate(bc)]
        return m
    if kind == "hexprism":
        return meshgen.hexprism_mesh(5, 4, 4, jitter=0.1, seed=2)
    return meshgen.merged_hex_mesh(6, 4, 4, jitter=0.1, seed=2)


def _scatter(n_cell, world, seed=7):
    rng = np.random.default_rng(seed)
    return rng.integers(0, world, n_cell).astype(np.int32)


@pytest.mark.parametrize("kind", ["box", "hexprism", "merged"])
@pytest.mark.parametrize("world,how", [(1, "slab"), (2, "slab"), (3, "slab"), (4, "scatter")])
def test_split_covers_the_mesh(kind, world, how):
    m = _mesh(kind)
    part_of = pa.slab_parts(m.n_cell, world) if how == "slab" else _scatter(m.n_cell, world)
    parts = pa.split(m, part_of, world)
    assert sorted(np.concatenate([p.cells for p in parts]).tolist()) == list(range(m.n_cell))
    assert sorted(np.concatenate([p.bfaces for p in parts]).tolist()) == list(range(m.n_bface))
    f2c = np.asarray(m.f2c).reshape(-1, 2)
    interior = f2c[m.n_bface:]
    n_cut = int(np.sum(part_of[interior[:, 0]] != part_of[interior[:, 1]]))
    assert sum(len(p.interfaces.nbz) for p in parts) == 2 * n_cut
    assert sum(p.mesh.n_face for p in parts) == m.n_face + n_cut
    for p in parts:
        lf = np.asarray(p.mesh.f2c).reshape(-1, 2)
        G = p.mesh.n_bface
        assert np.all(lf[:G, 1] < 0) and np.all(lf[G:, 1] >= 0) and np.all(lf[:, 0] >= 0)
        iface = lf[p.n_own_bface:G, 1]
        assert np.all(iface == -p.mesh.patches[-1][0])
        assert p.mesh.patches[-1][1] == meshgen.INTERFACE
        # the interface block names each face's partner, which names it back
        for k, (z, f) in enumerate(zip(p.interfaces.nbz, p.interfaces.nbf)):
            q = parts[z]
            j = f - q.n_own_bface
            assert q.interfaces.nbz[j] == p.rank and q.interfaces.nbf[j] == p.n_own_bface + k
            assert p.iface_cells[k] == q.cells[np.asarray(q.mesh.f2c)[2 * f]]
        # shared nodes: the same point on both sides
        it = p.interfaces
        for s, z, r in zip(it.nbsn, it.nbzn, it.nbrn):
            assert p.nodes[s] == parts[z].nodes[r]
    if world == 1:
        p = parts[0]
        for k in ("x", "y", "z", "nnpf", "f2n", "f2c"):
            assert np.array_equal(np.asarray(getattr(p.mesh, k)), np.asarray(getattr(m, k)))


@pytest.mark.parametrize("world", [1, 2, 3, 4, 7])
def test_rcb_parts_balanced_and_compact(world):
    m = meshgen.box_mesh(8, 6, 5, jitter=0.1, seed=1)
    part_of = pa.rcb_parts(m, world)
    counts = np.bincount(part_of, minlength=world)
    assert counts.sum() == m.n_cell and counts.min() >= m.n_cell // world - world
    assert counts.max() - counts.min() <= world
    # far fewer cut faces than a random assignment
    f2c = np.asarray(m.f2c).reshape(-1, 2)[m.n_bface:]
    cut = np.sum(part_of[f2c[:, 0]] != part_of[f2c[:, 1]])
    rnd = _scatter(m.n_cell, world)
    cut_rnd = np.sum(rnd[f2c[:, 0]] != rnd[f2c[:, 1]])
    assert world == 1 and cut == 0 or cut < 0.25 * cut_rnd
    pts = pa.cell_points(m)
    assert pts.shape == (m.n_cell, 3) and np.all((pts > 0) & (pts < 1))


def test_split_rejects_bad_maps():
    m = _mesh()
    with pytest.raises(ValueError):
        pa.split(m, np.zeros(m.n_cell - 1, np.int32), 1)
    with pytest.raises(ValueError):
        pa.split(m, np.full(m.n_cell, 2, np.int32), 2)
    with pytest.raises(ValueError):
        pa.slab_parts(10, 0)
    with pytest.raises(ValueError):  # an empty part
        pa.split(m, np.zeros(m.n_cell, np.int32), 2)


@pytest.mark.parametrize("world,how", [(2, "slab"), (3, "scatter")])
def test_halo_lists_agree_between_neighbours(world, how):
    m = _mesh()
    part_of = pa.slab_parts(m.n_cell, world) if how == "slab" else _scatter(m.n_cell, world)
    parts = pa.split(m, part_of, world)
    lists = [pa.halo_lists(p.mesh, p.interfaces, p.rank) for p in parts]
    for p, hl in zip(parts, lists):
        assert hl.row_ptr[-1] == hl.send_cells.size == hl.recv_bfaces.size
        for k, r in enumerate(hl.neighbors):
            q, ql = parts[r], lists[r]
            j = ql.neighbors.index(p.rank)
            a, b = slice(hl.row_ptr[k], hl.row_ptr[k + 1]), slice(ql.row_ptr[j], ql.row_ptr[j + 1])
            # what p sends to r lands where r expects it, and the reverse
            sent = p.cells[hl.send_cells[a]]
            expect = q.iface_cells[ql.recv_bfaces[b] - q.n_own_bface]
            assert np.array_equal(sent, expect)
            a, b = (slice(hl.node_ptr[k], hl.node_ptr[k + 1]),
                    slice(ql.node_ptr[j], ql.node_ptr[j + 1]))
            assert np.array_equal(p.nodes[hl.nodes[a]], q.nodes[ql.nodes[b]])


def test_part_grid_file_round_trip(tmp_path):
    m = _mesh()
    parts = pa.split(m, pa.slab_parts(m.n_cell, 3), 3)
    p = parts[1]
    path = tmp_path / "zone1.mfl"
    flowstar.write_grid(p.mesh, path, p.interfaces)
    back, itf = flowstar.read_grid(path)
    for k in ("x", "y", "z", "nnpf", "f2n", "f2c"):
        assert np.array_equal(np.asarray(getattr(back, k)), np.asarray(getattr(p.mesh, k)))
    assert back.n_bface == p.mesh.n_bface
    for k in ("nbz", "nbf", "nbsn", "nbzn", "nbrn"):
        assert np.array_equal(getattr(itf, k), getattr(p.interfaces, k))
    a = pa.halo_lists(back, itf, 1)
    b = pa.halo_lists(p.mesh, p.interfaces, 1)
    for k in ("send_cells", "recv_bfaces", "nodes", "row_ptr", "node_ptr"):
        assert np.array_equal(getattr(a, k), getattr(b, k))


def test_part_preprocessing_matches_whole_mesh():
    m = _mesh()
    params = gr.make_params(mach=0.6, alpha=3.0, cfl_start=10.0)
    parts = pa.split(m, _scatter(m.n_cell, 3), 3)
    whole, pgs = pa.prepare_parts(m, params, parts, bump_amp=0.05, bump_sigma=0.2)
    W = whole.arrays
    for pt, pg in zip(parts, pgs):
        A = pg.arrays
        C = pt.cells.size
        for k in ("vol", "xcc", "ycc", "zcc"):
            np.testing.assert_allclose(A[k][:C], W[k][pt.cells], rtol=1e-12, atol=1e-15)
        # a face keeps its area; one turned round reverses its normal
        lf = np.asarray(pt.mesh.f2c).reshape(-1, 2)
        for k in range(pt.n_own_bface, pt.mesh.n_bface):
            inner = pt.cells[lf[k, 0]]
            outer = pt.iface_cells[k - pt.n_own_bface]
            g = np.nonzero(((whole.arrays["f2c"][0::2] == inner) &
                            (whole.arrays["f2c"][1::2] == outer)) |
                           ((whole.arrays["f2c"][0::2] == outer) &
                            (whole.arrays["f2c"][1::2] == inner)))[0]
            assert g.size == 1
            g = g[0]
            sign = 1.0 if whole.arrays["f2c"][2 * g] == inner else -1.0
            np.testing.assert_allclose(A["area"][k], W["area"][g], rtol=1e-13)
            for n in ("xfn", "yfn", "zfn"):
                np.testing.assert_allclose(A[n][k], sign * W[n][g], rtol=1e-12, atol=1e-14)
        # the initial state: cells and every ghost from the whole mesh
        q = pg.q0.reshape(5, -1)
        Q = whole.q0.reshape(5, -1)
        assert np.array_equal(q[:, :C], Q[:, pt.cells])
        assert np.array_equal(q[:, C:C + pt.n_own_bface], Q[:, whole.n_cell + pt.bfaces])
        assert np.array_equal(q[:, C + pt.n_own_bface:], Q[:, pt.iface_cells])
        assert np.array_equal(A["nmark"], W["nmark"][pt.nodes])


def _zone_case(world, how, seed=7):
    m = _mesh()
    params = gr.make_params(mach=0.6, alpha=3.0, cfl_start=10.0)
    part_of = {"slab": lambda: pa.slab_parts(m.n_cell, world),
               "scatter": lambda: _scatter(m.n_cell, world, seed),
               "rcb": lambda: pa.rcb_parts(m, world)}[how]()
    parts = pa.split(m, part_of, world)
    return m, params, parts


def _compare_node_data(pt, A, W):
    # marks and flags exactly; sums to round-off (a cell next to a cut has
    # its faces in another order, so its centroid and weights may differ in
    # the last bit)
    assert np.array_equal(A["nmark"], W["nmark"])
    assert np.array_equal(A["nodesymm"], W["nodesymm"])
    np.testing.assert_allclose(A["wnode"], W["wnode"], rtol=1e-14)
    for k in ("xfn_n_symm", "yfn_n_symm", "zfn_n_symm"):
        np.testing.assert_allclose(A[k], W[k], rtol=1e-14, atol=1e-15)


@pytest.mark.parametrize("world,how", [(2, "slab"), (3, "scatter"), (4, "rcb")])
def test_zone_node_data_from_zone_grids_alone(world, how):
    m, params, parts = _zone_case(world, how)
    _, restricted = pa.prepare_parts(m, params, parts, bump_amp=0.05, bump_sigma=0.2)
    pgs = {p.rank: gr.prepare(p.mesh, params, bump_amp=0.05, bump_sigma=0.2) for p in parts}
    lists = {p.rank: pa.halo_lists(p.mesh, p.interfaces, p.rank) for p in parts}
    # on its own a zone misses the other zones' shares of its shared nodes
    assert all(not np.allclose(pgs[p.rank].arrays["wnode"], restricted[p.rank].arrays["wnode"])
               for p in parts)
    pa.zone_node_data(pgs, lists, pa.LocalExchange())
    for p in parts:
        _compare_node_data(p, pgs[p.rank].arrays, restricted[p.rank].arrays)


# ---- the exchanges on host buffers ------------------------------------------

def _fill(pt, buf, rank):
    """The packing restated: a sent row holds the whole-mesh id of its cell
    (and the sender); a node entry holds a partial sum that depends on the
    sender and the node."""
    hl = buf.lists
    rows = np.zeros((max(hl.send_cells.size, 1), 8))
    rows[:hl.send_cells.size, 0] = pt.cells[hl.send_cells]
    rows[:hl.send_cells.size, 1] = rank
    nodes = np.zeros((max(hl.nodes.size, 1), 8))
    g = pt.nodes[hl.nodes]
    for v in range(5):
        nodes[:hl.nodes.size, v] = g * 10.0 + v + 1000.0 * rank
    import torch
    buf.send_rows.copy_(torch.from_numpy(rows))
    buf.node_send.copy_(torch.from_numpy(nodes))
    buf.ext.copy_(torch.tensor([100 + rank, 50 - rank], dtype=torch.int64))


def _check(pt, buf, parts_all):
    hl = buf.lists
    r = buf.recv_rows.numpy()
    nr = hl.recv_bfaces.size
    assert np.array_equal(r[:nr, 0], pt.iface_cells[hl.recv_bfaces - pt.n_own_bface])
    owners = np.asarray(pt.interfaces.nbz)[hl.recv_bfaces - pt.n_own_bface]
    assert np.array_equal(r[:nr, 1], owners)
    nd = buf.node_recv.numpy()
    for k, z in enumerate(hl.neighbors):
        for e in range(hl.node_ptr[k], hl.node_ptr[k + 1]):
            g = pt.nodes[hl.nodes[e]]
            assert nd[e, 0] == g * 10.0 + 1000.0 * z


def _world_parts(world):
    m = _mesh()
    parts = pa.split(m, _scatter(m.n_cell, world, seed=11), world)
    return parts


def test_local_exchange_on_host_buffers():
    parts = _world_parts(3)
    bufs = {p.rank: pa.HaloBuffers(pa.halo_lists(p.mesh, p.interfaces, p.rank), "cpu")
            for p in parts}
    for p in parts:
        _fill(p, bufs[p.rank], p.rank)
    ex = pa.LocalExchange()
    ex.rows(bufs)
    ex.nodes(bufs)
    ex.extrema(bufs)
    for p in parts:
        _check(p, bufs[p.rank], parts)
        assert bufs[p.rank].ext.tolist() == [102, 48]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out_dir):
    import datetime

    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    parts = _world_parts(world)
    p = parts[rank]
    buf = pa.HaloBuffers(pa.halo_lists(p.mesh, p.interfaces, p.rank), "cpu")
    _fill(p, buf, rank)
    ex = pa.DistExchange()
    ex.rows({rank: buf})
    ex.nodes({rank: buf})
    ex.extrema({rank: buf})
    hist = ex.sum(torch.full((3, 5), float(rank + 1), dtype=torch.float64))
    _check(p, buf, parts)
    np.save(os.path.join(out_dir, f"r{rank}.npy"),
            np.concatenate([buf.ext.numpy().astype(np.float64), hist.numpy().reshape(-1)]))
    dist.barrier()
    dist.destroy_process_group()


def _zone_rank_main(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    m, params, parts = _zone_case(world, "rcb")
    p = parts[rank]
    pg = gr.prepare(p.mesh, params)
    pa.zone_node_data({rank: pg}, {rank: pa.halo_lists(p.mesh, p.interfaces, rank)},
                      pa.DistExchange())
    np.savez(os.path.join(out_dir, f"z{rank}.npz"),
             **{k: pg.arrays[k] for k in ("wnode", "nmark", "nodesymm", "xfn_n_symm",
                                          "yfn_n_symm", "zfn_n_symm")})
    dist.barrier()
    dist.destroy_process_group()


def test_zone_node_data_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.spawn(_zone_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world,
             join=True)
    m, params, parts = _zone_case(world, "rcb")
    _, restricted = pa.prepare_parts(m, params, parts)
    for p in parts:
        got = dict(np.load(tmp_path / f"z{p.rank}.npz"))
        _compare_node_data(p, got, restricted[p.rank].arrays)


def test_dist_exchange_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    for r in range(world):
        v = np.load(tmp_path / f"r{r}.npy")
        assert v[:2].tolist() == [101.0, 49.0]
        assert np.all(v[2:] == 3.0)
