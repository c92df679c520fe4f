"""One mesh over several contexts (mfg_halo_set / mfg_halo_phase, the
reference's MPI mode) on one GPU, the parts exchanging by device copies:
one part against the fused single-mesh iteration bit for bit; several parts
against the whole mesh -- the initial gradient and the first residual to
round-off, the converged state to the convergence level -- and the
refusals."""
import ctypes as ct

import numpy as np
import pytest

from helpers import assert_bitwise
from minifs_b200 import _lib, flowstar, grid as gr, meshgen
from minifs_b200 import partition as pa
from minifs_b200.compare import state_rel_err
from minifs_b200.solver import Solver

pytestmark = pytest.mark.gpu

BC = (3, 6, 4, 61, 5, 6)


def _box(n=8):
    m = meshgen.box_mesh(n, n - 1, n - 2, jitter=0.2, seed=3, bc_types=BC)
    m.patches = [(i + 1, t) for i, t in enumerate(BC)]
    return m


def _params():
    return gr.make_params(mach=0.6, alpha=4.0, cfl_start=10.0)


BUMP = dict(bump_amp=0.05, bump_sigma=0.2)


def _whole(m, p, live=False):
    s = Solver(gr.prepare(m, p, **BUMP), p)
    if live:
        s.set_live_bc(True)
    return s


def _decomposed(m, p, world, part_of=None, live=False):
    parts, whole, held = pa.build_parts(m, p, world, part_of=part_of, **BUMP)
    if live:
        for hp in held.values():
            hp.solver.set_live_bc(True)
    return parts, whole, pa.Decomposed(held)


def _cells(parts, d, field, n_cell):
    return pa.assemble(parts, [d.download(field)[z] for z in sorted(d.parts)], n_cell)


def _scatter(n_cell, world, seed=5):
    return np.random.default_rng(seed).integers(0, world, n_cell).astype(np.int32)


def test_one_part_is_the_fused_iteration():
    m, p = meshgen.cube_mesh(8, jitter=0.15, seed=9), _params()
    ref = _whole(m, p)
    nref = ref.iterate(7)
    parts, _, d = _decomposed(m, p, 1)
    nd = d.iterate(7)
    s = d.parts[0].solver
    for f in ("q", "res", "dq", "dqdx", "dqdy", "dqdz", "dt"):
        assert_bitwise(s.download(f), ref.download(f), f"one part {f}")
    assert_bitwise(nd.reshape(-1), nref.reshape(-1), "norms")


@pytest.mark.parametrize("world,how", [(2, "slab"), (3, "scatter"), (4, "scatter")])
def test_initial_gradient_and_first_residual(world, how):
    m, p = _box(), _params()
    part_of = None if how == "slab" else _scatter(m.n_cell, world)
    parts, whole, d = _decomposed(m, p, world, part_of)
    ref = _whole(m, p)
    ref.calculate_gradient()
    C = whole.n_cell
    for f in ("dqdx", "dqdy", "dqdz"):
        g = _cells(parts, d, f, C)
        r = ref.download(f).reshape(5, -1)[:, :C]
        for v in range(5):
            scale = np.abs(r[v]).max() + 1e-300
            np.testing.assert_allclose(g[v], r[v], rtol=0, atol=1e-11 * scale,
                                       err_msg=f"{f}[{v}] {world} parts")
    n1 = d.iterate(1)
    nr = ref.iterate(1)
    res = _cells(parts, d, "res", C)
    rr = ref.download("res").reshape(5, -1)
    for v in range(5):
        scale = np.abs(rr[v]).max()
        np.testing.assert_allclose(res[v], rr[v], rtol=0, atol=1e-12 * scale)
    np.testing.assert_allclose(n1, nr, rtol=1e-11)
    dt = pa.assemble(parts, [d.download("dt")[z] for z in sorted(d.parts)], C, width=1)
    np.testing.assert_allclose(dt[0], ref.download("dt"), rtol=1e-12)


def _to_drop(run, drop, cap, chunk=100):
    """Iterate in chunks until the density residual fell by `drop`; returns
    (norms, iterations)."""
    norms = run(chunk)
    while norms[-1, 0] >= drop * norms[0, 0] and len(norms) < cap:
        norms = np.concatenate([norms, run(chunk)])
    return norms, len(norms)


@pytest.mark.parametrize("world,how,live", [(2, "slab", False), (4, "rcb", False),
                                            (3, "slab", True), (4, "scatter", False)])
def test_parts_converge_to_the_whole_mesh_state(world, how, live):
    m, p = _box(), _params()
    part_of = {"slab": None, "rcb": pa.rcb_parts(m, world),
               "scatter": _scatter(m.n_cell, world, seed=8)}[how]
    parts, whole, d = _decomposed(m, p, world, part_of, live)
    ref = _whole(m, p, live)
    # a scattered partition cuts nearly every face, and the sweeps' coupling
    # across parts is that of block Jacobi on single cells: more iterations
    nd, it_d = _to_drop(d.iterate, 1e-10, 4000)
    nr, it_r = _to_drop(ref.iterate, 1e-10, 4000)
    print(f"\n{world} parts ({how}{', live BC' if live else ''}): drop 1e-10 in {it_d} "
          f"iterations, the whole mesh in {it_r}")
    assert np.all(np.isfinite(nd))
    assert nd[-1, 0] < 1e-10 * nd[0, 0] and nr[-1, 0] < 1e-10 * nr[0, 0], (it_d, it_r)
    C = whole.n_cell
    q = _cells(parts, d, "q", C)
    Q = ref.download("q").reshape(5, -1)[:, :C]
    full = np.zeros((5, whole.n))
    full[:, :C] = q
    ref_full = np.zeros((5, whole.n))
    ref_full[:, :C] = Q
    err = state_rel_err(full.reshape(-1), ref_full.reshape(-1), whole.n, p.p_bar)["max_norm"]
    assert err < 1e-7, err
    # the parts did not follow the single mesh's path (block Jacobi across cuts)
    assert not np.allclose(nd[5], nr[5], rtol=1e-6)
    d.close()


def test_zones_from_their_own_files(tmp_path):
    """Each zone written as a FlowStar grid with its interface block and its
    bc.para, read back and set up from that alone (node data combined over
    the zones by exchange), against the zones set up from the whole mesh."""
    m, p = _box(), _params()
    world = 3
    parts, whole, held = pa.build_parts(m, p, world, part_of=pa.rcb_parts(m, world), **BUMP)
    ref = pa.Decomposed(held)
    zones = {}
    for pt in parts:
        g, b = tmp_path / f"zone{pt.rank}.mfl", tmp_path / f"zone{pt.rank}.bc"
        flowstar.write_grid(pt.mesh, g, pt.interfaces)
        flowstar.write_bc(pt.mesh.patches, b)
        mesh, itf = flowstar.read_grid(g)
        mesh.patches = flowstar.read_bc(b)
        zones[pt.rank] = (mesh, itf)
    d = pa.Decomposed(pa.build_zones(zones, p, **BUMP))
    C = whole.n_cell
    for f in ("dqdx", "dqdy", "dqdz"):
        a, b = _cells(parts, d, f, C), _cells(parts, ref, f, C)
        for v in range(5):
            np.testing.assert_allclose(a[v], b[v], rtol=0, atol=1e-11 * np.abs(b[v]).max())
    na, nb = d.iterate(40), ref.iterate(40)
    np.testing.assert_allclose(na, nb, rtol=1e-9)
    qa, qb = _cells(parts, d, "q", C), _cells(parts, ref, "q", C)
    for v in range(5):
        np.testing.assert_allclose(qa[v], qb[v], rtol=1e-10, atol=1e-10 * np.abs(qb[v]).max())
    d.close()
    ref.close()


@pytest.mark.parametrize("order", [2, 3, 4])
def test_second_order_across_parts(order):
    """At second order the interface ghosts' face states are reconstructed
    from the neighbouring cells' gradients, limiters and centroids: the
    first residual and limiter of 3 parts equal the whole mesh's to
    round-off (a first-order ghost would leave the cut faces' fluxes off
    by the reconstruction itself)."""
    m, p = _box(), _params()
    world = 3
    parts, whole, held = pa.build_parts(m, p, world, part_of=pa.rcb_parts(m, world), **BUMP)
    d = pa.Decomposed(held)
    ref = _whole(m, p)
    ref.set_order(order)
    d.set_order(order)
    nr, nd = ref.iterate(1), d.iterate(1)
    C = whole.n_cell
    res, rr = _cells(parts, d, "res", C), ref.download("res").reshape(5, -1)
    for v in range(5):
        np.testing.assert_allclose(res[v], rr[v], rtol=0, atol=1e-11 * np.abs(rr[v]).max(),
                                   err_msg=f"order {order} res[{v}]")
    np.testing.assert_allclose(nd, nr, rtol=1e-10)
    if order >= 3:
        lim = pa.assemble(parts, [d.download("limiter")[z] for z in sorted(d.parts)], C)
        off = np.abs(lim - ref.download("limiter").reshape(5, -1)) > 1e-9
        if order == 4:  # Venkatakrishnan's limiter is smooth
            assert not off.any()
        else:
            # Barth's min(1, d1/d2) jumps where d2 = grad q . r changes sign
            # (a face nearly along an isoline of a cell that is a local
            # extremum): round-off in the gradient decides it at a few cells
            assert off.mean() < 1e-3, off.sum()
    n2 = d.iterate(20)
    assert np.all(np.isfinite(n2)) and n2[-1, 0] < n2[0, 0]
    d.close()


def test_mixed_form_across_parts():
    """The mixed form (single-precision dissipation, gradient and off-diagonal
    LU-SGS products; node partial sums exchanged in single precision): one
    part is the fused mixed iteration bit for bit; 3 parts stay within the
    mixed form's own rounding of the whole mesh's mixed iterations."""
    m, p = _box(), _params()
    _, _, held1 = pa.build_parts(m, p, 1, precision="mixed", **BUMP)
    hp = held1[0]
    d1 = pa.Decomposed(held1)
    ref = Solver(gr.prepare(m, p, **BUMP), p, precision="mixed")
    nr = ref.iterate(6)
    n1 = d1.iterate(6)
    for f in ("q", "res", "dq", "dqdx"):
        assert_bitwise(hp.solver.download(f), ref.download(f), f"mixed one part {f}")
    assert_bitwise(n1.reshape(-1), nr.reshape(-1), "mixed norms")
    d1.close()
    world = 3
    parts, whole, held = pa.build_parts(m, p, world, part_of=pa.rcb_parts(m, world),
                                        precision="mixed", **BUMP)
    d = pa.Decomposed(held)
    ref = Solver(gr.prepare(m, p, **BUMP), p, precision="mixed")
    ref.calculate_gradient()
    C = whole.n_cell
    g, r = _cells(parts, d, "dqdx", C), ref.download("dqdx").reshape(5, -1)[:, :C]
    for v in range(5):
        np.testing.assert_allclose(g[v], r[v], rtol=0, atol=1e-5 * np.abs(r[v]).max())
    nd, nr = d.iterate(1), ref.iterate(1)
    np.testing.assert_allclose(nd, nr, rtol=1e-6)
    nd, it_d = _to_drop(d.iterate, 1e-6, 3000)
    assert np.all(np.isfinite(nd)) and nd[-1, 0] < 1e-6 * nd[0, 0], it_d
    d.close()


def test_halo_refusals_and_checks():
    m, p = _box(6), _params()
    parts, whole, d = _decomposed(m, p, 2)
    s = d.parts[0].solver
    for call in (lambda: s.iterate(1), lambda: s.calculate_gradient(),
                 lambda: s.forward_lusgs()):
        with pytest.raises(_lib.MfgError) as e:
            call()
        assert e.value.code == -6
    lib = s.lib
    assert lib.mfg_halo_phase(s.ctx, 99, 0) == -1
    plain = Solver(gr.prepare(m, p, **BUMP), p)
    assert lib.mfg_halo_phase(plain.ctx, 1, 0) == -6  # no halo registered
    # a received row must fill the ghost of an interface face
    import torch
    buf = pa.HaloBuffers(pa.HaloLists(rank=0, neighbors=[], send_cells=np.zeros(0, np.int32),
                                      recv_bfaces=np.zeros(1, np.int32),
                                      nodes=np.zeros(0, np.int32), row_ptr=np.zeros(1),
                                      node_ptr=np.zeros(1)), torch.device("cuda", 0))
    h = _lib.Halo()
    rb = np.zeros(1, np.int32)  # boundary face 0 is a wall of the whole mesh
    h.n_recv, h.recv_bfaces = 1, _lib.ptr(rb, _lib.i32p)
    for name in ("send_rows", "recv_rows", "node_send", "node_recv", "ext", "norm_sq"):
        setattr(h, name, ct.c_void_p(getattr(buf, name).data_ptr()))
    assert lib.mfg_halo_set(plain.ctx, ct.byref(h)) == -1
    # second order without the gradient rows' buffers
    second = Solver(gr.prepare(m, p, **BUMP), p)
    second.set_order(3)
    rb2 = np.array([parts[0].n_own_bface], np.int32)
    h.recv_bfaces = _lib.ptr(rb2, _lib.i32p)
    assert lib.mfg_halo_set(second.ctx, ct.byref(h)) == -6
    from minifs_b200.solver import BatchSolver
    batch = BatchSolver([gr.prepare(m, p, **BUMP)] * 2, [p, p])
    h.n_recv = 0
    assert lib.mfg_halo_set(batch.ctx, ct.byref(h)) == -6  # one case per context
    d.close()
