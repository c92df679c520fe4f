"""Second-order reconstruction (mfg_set_order: the reference's `order` switch,
which it declares but does not implement): the GPU residual and limiter
against a NumPy restatement of the same reconstruction and limiters around
the oracle's Roe flux, bit for bit; the properties the limiters promise;
freestream preservation; convergence."""
import math

import numpy as np
import pytest

from helpers import assert_bitwise
from minifs_b200 import grid as gr, meshgen
from minifs_b200.compare import state_rel_err
from minifs_b200.solver import Solver
from oracle import oracle_py

pytestmark = pytest.mark.gpu


def _case(n=8, bump=0.05, mesh=None):
    m = mesh if mesh is not None else meshgen.cube_mesh(n, jitter=0.15, seed=9)
    p = gr.make_params(mach=0.6, alpha=3.0, cfl_start=10.0)
    pg = gr.prepare(m, p, bump_amp=bump, bump_sigma=0.15)
    return m, p, pg


def _limiter(order, pg, q, gx, gy, gz, k=5.0):
    """phi[5][C] as the limiter kernel forms it."""
    a = pg.arrays
    C, G, n = pg.n_cell, pg.n_bface, pg.n
    f2c = np.asarray(a["f2c"])
    xcc, ycc, zcc = (np.asarray(a[t]) for t in ("xcc", "ycc", "zcc"))
    xfc, yfc, zfc = (np.asarray(a[t]) for t in ("xfc", "yfc", "zfc"))
    # the C library's cbrt, as the library's host code evaluates h
    h = [math.cbrt(abs(v)) for v in np.asarray(a["vol"])[:C].tolist()]
    Q = q.reshape(5, n)
    phi = np.ones((5, C))
    qmin = Q[:, :C].copy()
    qmax = Q[:, :C].copy()
    faces_of = [[] for _ in range(C)]
    for f in range(pg.n_face):
        c1, c2 = int(f2c[2 * f]), int(f2c[2 * f + 1])
        faces_of[c1].append((f, c2))
        if f >= G:
            faces_of[c2].append((f, c1))
    for c in range(C):
        for _, nb in faces_of[c]:
            qmin[:, c] = np.minimum(qmin[:, c], Q[:, nb])
            qmax[:, c] = np.maximum(qmax[:, c], Q[:, nb])
        eps2 = (k * h[c]) * (k * h[c]) * (k * h[c]) if order == 4 else 0.0
        for f, _ in faces_of[c]:
            rx, ry, rz = xfc[f] - xcc[c], yfc[f] - ycc[c], zfc[f] - zcc[c]
            for v in range(5):
                i = v * n + c
                d2 = gx[i] * rx + gy[i] * ry + gz[i] * rz
                if d2 == 0.0:
                    continue
                d1 = (qmax[v, c] if d2 > 0.0 else qmin[v, c]) - Q[v, c]
                if order == 4:
                    aa = d1 * d1 + eps2
                    psi = (aa + 2.0 * d2 * d1) / (aa + 2.0 * d2 * d2 + d1 * d2)
                else:
                    psi = min(1.0, d1 / d2)
                phi[v, c] = min(phi[v, c], psi)
    return np.maximum(0.0, np.minimum(1.0, phi)), qmin, qmax


def _residual(order, pg, p, q, gx, gy, gz, phi):
    """The residual of one flux evaluation with reconstructed face states."""
    a = pg.arrays
    C, G, n = pg.n_cell, pg.n_bface, pg.n
    f2c = np.asarray(a["f2c"])
    Q = q.reshape(5, n)
    res = np.zeros((5, C))
    cen = {t: np.asarray(a[t]) for t in ("xcc", "ycc", "zcc", "xfc", "yfc", "zfc")}

    def rec(c, f):
        s = Q[:, c].copy()
        if c >= C:
            return s
        rx = cen["xfc"][f] - cen["xcc"][c]
        ry = cen["yfc"][f] - cen["ycc"][c]
        rz = cen["zfc"][f] - cen["zcc"][c]
        for v in range(5):
            i = v * n + c
            d = gx[i] * rx + gy[i] * ry + gz[i] * rz
            s[v] = s[v] + (phi[v, c] if phi is not None else 1.0) * d
        return s

    for f in range(pg.n_face):
        c1, c2 = int(f2c[2 * f]), int(f2c[2 * f + 1])
        ql, qr = rec(c1, f), rec(c2, f)
        if not (ql[0] > 0.0 and qr[0] > 0.0 and ql[4] + p.p_bar > 0.0 and qr[4] + p.p_bar > 0.0):
            ql, qr = Q[:, c1].copy(), Q[:, c2].copy()
        fl = oracle_py.roe_flux(ql, qr, (a["xfn"][f], a["yfn"][f], a["zfn"][f]), a["area"][f],
                                p.gam, p.gamm1, p.p_bar, p.alf_l)
        res[:, c1] -= fl
        if c2 < C:
            res[:, c2] += fl
    return res.reshape(-1)


@pytest.mark.parametrize("order", [2, 3, 4])
def test_residual_and_limiter_match_restatement(order):
    m, p, pg = _case()
    s = Solver(pg, p)
    s.iterate(3)  # a state with gradients
    s.set_order(order)
    q = s.download("q")
    gx, gy, gz = s.download("dqdx"), s.download("dqdy"), s.download("dqdz")
    s.zero_residuals()
    s.inviscid_flux()
    res = s.download("res")
    phi = None
    if order >= 3:
        phi, _, _ = _limiter(order, pg, q, gx, gy, gz)
        assert_bitwise(s.download("limiter"), phi.reshape(-1), f"order {order} limiter")
    assert_bitwise(res, _residual(order, pg, p, q, gx, gy, gz, phi), f"order {order} residual")
    first = Solver(pg, p)
    first.upload_q(q)
    first.zero_residuals()
    first.inviscid_flux()
    assert not np.array_equal(first.download("res"), res)  # the reconstruction acts


def test_barth_keeps_face_values_in_range():
    m, p, pg = _case()
    s = Solver(pg, p)
    s.iterate(3)
    s.set_order(3)
    s.zero_residuals()
    s.inviscid_flux()
    q = s.download("q")
    gx, gy, gz = s.download("dqdx"), s.download("dqdy"), s.download("dqdz")
    phi = s.download("limiter").reshape(5, pg.n_cell)
    _, qmin, qmax = _limiter(3, pg, q, gx, gy, gz)
    a, C, G, n = pg.arrays, pg.n_cell, pg.n_bface, pg.n
    f2c = np.asarray(a["f2c"])
    Q = q.reshape(5, n)
    assert phi.min() >= 0.0 and phi.max() <= 1.0 and phi.min() < 1.0
    for f in range(pg.n_face):
        for c in (int(f2c[2 * f]), int(f2c[2 * f + 1])):
            if c >= C:
                continue
            r = (a["xfc"][f] - a["xcc"][c], a["yfc"][f] - a["ycc"][c], a["zfc"][f] - a["zcc"][c])
            for v in range(5):
                i = v * n + c
                val = Q[v, c] + phi[v, c] * (gx[i] * r[0] + gy[i] * r[1] + gz[i] * r[2])
                scale = abs(qmax[v, c]) + abs(qmin[v, c]) + (p.p_bar if v == 4 else 1.0)
                assert qmin[v, c] - 1e-12 * scale <= val <= qmax[v, c] + 1e-12 * scale


@pytest.mark.parametrize("order", [2, 3, 4])
def test_freestream_preserved(order):
    m, p, pg = _case(bump=0.0)
    s = Solver(pg, p)
    s.set_order(order)
    q0 = s.download("q")
    s.iterate(5)
    err = state_rel_err(s.download("q"), q0, pg.n, p.p_bar)["max_norm"]
    assert err < 1e-10, err


@pytest.mark.parametrize("order", [3, 4])
def test_second_order_converges(order):
    m, p, pg = _case(n=12)
    s = Solver(pg, p)
    s.set_order(order)
    nrm = s.iterate(600)
    assert np.all(np.isfinite(nrm))
    assert nrm[-1, 0] < 1e-3 * nrm[0, 0], nrm[-1, 0] / nrm[0, 0]
    # the fused path equals the per-routine path under second order
    a, b = Solver(pg, p), Solver(pg, p)
    for x in (a, b):
        x.set_order(order)
    a.iterate(4)
    for _ in range(4):
        b.step()
    assert_bitwise(a.download("q"), b.download("q"), "fused vs per routine")


def test_mixed_form_second_order_close_to_fp64():
    m, p, pg = _case()
    a, b = Solver(pg, p), Solver(pg, p, precision="mixed")
    for x in (a, b):
        x.set_order(4)
        x.iterate(10)
    assert state_rel_err(b.download("q"), a.download("q"), pg.n, p.p_bar)["max_norm"] < 1e-6
