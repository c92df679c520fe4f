"""Known answers of single reference functions (tests/golden/make_kats.py:
RoeFlux_noprec, cal_flux.cpp:301-834, FluxLUSGS3D,
forward_lusgs.cpp:1271-1324, and UpdateFlowField3D_CFL3d,
forward_lusgs.cpp:1335-1488, called directly on inputs chosen to reach the
entropy fix's branches, sonic and supersonic faces, strong jumps, equal
states, axis-aligned normals, zero increments, the update's density and
pressure relaxation and its clamps) against the CPU oracle's functions:
bit for bit."""
import os

import numpy as np
import pytest

from helpers import assert_bitwise

HERE = os.path.dirname(os.path.abspath(__file__))
GROUPS = ("random", "stagnation", "sonic", "supersonic", "jump", "equal", "axis")


@pytest.fixture(scope="module")
def kats():
    return dict(np.load(os.path.join(HERE, "golden", "kats.npz")))


@pytest.mark.parametrize("s", [0, 1])
def test_roe_flux_matches_reference(kats, s):
    from oracle import oracle_py
    _, epsa_r, _, gam, p_bar = kats[f"s{s}_params"]
    ql, qr, nrm, area = (kats[f"s{s}_{k}"] for k in ("ql", "qr", "normal", "area"))
    ref, grp = kats[f"s{s}_roe_flux"], kats[f"s{s}_group"]
    got = np.stack([oracle_py.roe_flux(ql[:, f], qr[:, f], nrm[f], area[f], gam, gam - 1.0,
                                       p_bar, epsa_r) for f in range(ql.shape[1])], axis=1)
    assert np.isfinite(ref).all()
    for g, name in enumerate(GROUPS):
        sel = grp == g
        assert sel.sum() > 0, name
        assert_bitwise(got[:, sel].ravel(), ref[:, sel].ravel(), f"set {s} {name}")
    if epsa_r > 0:
        # the groups reach the branches they are meant to: without the
        # entropy fix every stagnation and sonic face changes, no supersonic
        # face does
        def fixed(f):
            nofix = oracle_py.roe_flux(ql[:, f], qr[:, f], nrm[f], area[f], gam, gam - 1.0,
                                       p_bar, 0.0)
            return not np.array_equal(got[:, f], nofix)
        for name, want in (("stagnation", True), ("sonic", True), ("supersonic", False)):
            faces = np.nonzero(grp == GROUPS.index(name))[0]
            assert all(fixed(f) == want for f in faces), name


@pytest.mark.parametrize("s", [0, 1])
def test_flux_lusgs_matches_reference(kats, s):
    from oracle import oracle_py
    _, _, lhs, gam, p_bar = kats[f"s{s}_params"]
    cases, ref = kats[f"s{s}_lusgs_in"], kats[f"s{s}_lusgs_flux"]
    got = np.stack([oracle_py.flux_lusgs(c[:5], c[5:10], c[10:13], gam, p_bar, lhs)
                    for c in cases])
    assert np.isfinite(ref).all()
    assert (np.abs(cases[:, 5:10]).sum(1) == 0).any()  # zero increments are among the cases
    assert_bitwise(got.ravel(), ref.ravel(), f"set {s} FluxLUSGS3D")


UPDATE_GROUPS = ("small", "rho_drop", "p_drop", "both_drop", "rho_high", "p_high")


@pytest.mark.parametrize("s", [0, 1])
def test_update_flow_matches_reference(kats, s):
    from oracle import oracle_py
    _, _, _, gam, p_bar = kats[f"s{s}_params"]
    rho_s, rho_min, rho_max, p_min, p_max = kats[f"s{s}_update_limits"]
    q, dq, grp = kats[f"s{s}_update_q"], kats[f"s{s}_update_dq"], kats[f"s{s}_update_group"]
    ref = kats[f"s{s}_update_out"]
    got = oracle_py.update_flow(q, dq, dict(gam=gam, p_bar=p_bar, rho_s=rho_s, rho_min=rho_min,
                                            rho_max=rho_max, p_min=p_min, p_max=p_max))
    for g, name in enumerate(UPDATE_GROUPS):
        sel = grp == g
        assert_bitwise(got[:, sel].ravel(), ref[:, sel].ravel(), f"set {s} update {name}")
    # the groups reach their branches: relaxed density drops are smaller
    # than the raw increment, and the high groups end on the clamps
    sel = (grp == 1) | (grp == 3)
    assert (ref[0, sel] > q[0, sel] + dq[0, sel]).all()
    assert (ref[0, grp == 4] == rho_max).all()
    assert (ref[4, grp == 5] == p_max).all()
