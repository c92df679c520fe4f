"""Known answers of single reference functions on the GPU: the fixture of
tests/golden/kats.npz (RoeFlux_noprec, cal_flux.cpp:676-834, FluxLUSGS3D,
forward_lusgs.cpp:1271-1324, UpdateFlowField3D_CFL3d,
forward_lusgs.cpp:1335-1488, each called directly by the reference on
inputs that reach the entropy fix at stagnation and sonic faces,
supersonic faces, strong jumps, equal states, axis normals, zero
increments, the density and pressure relaxation and the clamps) run
through the device functions the iteration kernels use, via the
mfg_selftest_functions hook: bit for bit against the reference's outputs.
The mesh parity cases need not reach every one of these branches."""
import ctypes as ct
import os

import numpy as np
import pytest

from helpers import assert_bitwise

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GROUPS = ("random", "stagnation", "sonic", "supersonic", "jump", "equal", "axis")
UPDATE_GROUPS = ("small", "rho_drop", "p_drop", "both_drop", "rho_high", "p_high")


@pytest.fixture(scope="module")
def kats():
    return dict(np.load(os.path.join(HERE, "golden", "kats.npz")))


@pytest.fixture(scope="module")
def lib():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from minifs_b200 import _lib
    return _lib.load()


def _run(lib, mode, n, consts, inp):
    f64p = ct.POINTER(ct.c_double)
    consts = np.ascontiguousarray(consts, np.float64)
    inp = np.ascontiguousarray(inp, np.float64)
    out = np.zeros(5 * n)
    rc = lib.mfg_selftest_functions(mode, n, consts.ctypes.data_as(f64p),
                                    inp.ctypes.data_as(f64p), out.ctypes.data_as(f64p))
    assert rc == 0, lib.mfg_last_cuda_error()
    return out


def _consts(kats, s, limits=(0.0, 0.0, 0.0, 0.0)):
    _, epsa_r, lhs, gam, p_bar = kats[f"s{s}_params"]
    return [gam, p_bar, epsa_r, lhs, *limits]


@pytest.mark.parametrize("s", [0, 1])
def test_roe_flux_device_matches_reference(kats, lib, s):
    ql, qr, nrm, area = (kats[f"s{s}_{k}"] for k in ("ql", "qr", "normal", "area"))
    F = ql.shape[1]
    inp = np.concatenate([ql.ravel(), qr.ravel(), nrm[:, 0], nrm[:, 1], nrm[:, 2], area])
    got = _run(lib, 0, F, _consts(kats, s), inp).reshape(5, F)
    ref, grp = kats[f"s{s}_roe_flux"], kats[f"s{s}_group"]
    for g, name in enumerate(GROUPS):
        sel = grp == g
        assert sel.sum() > 0, name
        assert_bitwise(got[:, sel].ravel(), ref[:, sel].ravel(), f"set {s} {name} (GPU)")


@pytest.mark.parametrize("mode", [1, 3])
@pytest.mark.parametrize("s", [0, 1])
def test_flux_lusgs_device_matches_reference(kats, lib, s, mode):
    """mode 1: the device FluxLUSGS3D; mode 3: the persistent sweeps' form
    with branch-free divisions."""
    cases, ref = kats[f"s{s}_lusgs_in"], kats[f"s{s}_lusgs_flux"]
    got = _run(lib, mode, cases.shape[0], _consts(kats, s), cases).reshape(-1, 5)
    assert_bitwise(got.ravel(), ref.ravel(), f"set {s} FluxLUSGS3D mode {mode} (GPU)")


@pytest.mark.parametrize("s", [0, 1])
def test_update_flow_device_matches_reference(kats, lib, s):
    _, rho_min, rho_max, p_min, p_max = kats[f"s{s}_update_limits"]
    q, dq, grp = kats[f"s{s}_update_q"], kats[f"s{s}_update_dq"], kats[f"s{s}_update_group"]
    C = q.shape[1]
    got = _run(lib, 2, C, _consts(kats, s, (rho_min, rho_max, p_min, p_max)),
               np.concatenate([q.ravel(), dq.ravel()])).reshape(5, C)
    ref = kats[f"s{s}_update_out"]
    for g, name in enumerate(UPDATE_GROUPS):
        sel = grp == g
        assert sel.sum() > 0, name
        assert_bitwise(got[:, sel].ravel(), ref[:, sel].ravel(), f"set {s} update {name} (GPU)")
