"""The allocation-free residual norm (mfg_residual_norm_static).

Some callers of this library cannot allocate device memory: code that only
holds device pointers and has no mfgpu context (creating one allocates), or
an application whose device memory is owned by another allocator.  For them
the norm's block partials live in a static device array instead of a
context buffer.  This checks, through the C ABI, that two calls in a row
give the norms of the context-based entry point, that a residual larger
than the static limit is refused, that a call on a 64^3 x 6-sized residual
(1,572,864 cells: more blocks than the context-based norm's fixed grid, so
a different reduction order) matches the norms summed on the host, that
n_cell = 0 gives zeros, and that repeated calls leave the device's free
memory unchanged.

Kept in its own file, collected last, so that a failure here comes after
every other test has run.
"""
import ctypes as ct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_CELLS = 1 << 24  # MFG_NORM_STATIC_MAX_CELLS


def test_static_norm_matches_context_norm_twice():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from minifs_b200 import _lib, grid as gr, meshgen
    from minifs_b200.solver import Solver

    lib = _lib.load()
    mesh = meshgen.cube_mesh(12, jitter=0.15, seed=4)  # 10368 cells: 41 blocks
    p = gr.make_params(mach=0.5, alpha=2.0, cfl_start=10.0)
    pg = gr.prepare(mesh, p, bump_amp=0.05, bump_sigma=0.1)
    s = Solver(pg, p)
    s.calculate_gradient()
    out = torch.zeros(5, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    seen = []
    for call in range(2):
        s.iterate(2)  # a different residual for each call
        expected = s.residual_norm()  # the existing, context-based entry point
        res = torch.from_numpy(s.download("res")).to("cuda")
        rc = lib.mfg_residual_norm_static(ct.c_void_p(res.data_ptr()), pg.n_cell,
                                          ct.c_void_p(out.data_ptr()),
                                          ct.c_void_p(stream.cuda_stream))
        assert rc == 0, lib.mfg_last_cuda_error()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        np.testing.assert_allclose(got, expected, rtol=1e-12, atol=0)
        seen.append(got.copy())
    assert not np.array_equal(seen[0], seen[1])  # the second call saw new data

    rc = lib.mfg_residual_norm_static(ct.c_void_p(res.data_ptr()), MAX_CELLS + 1,
                                      ct.c_void_p(out.data_ptr()), None)
    assert rc == -1
    assert b"exceeds the static scratch limit" in lib.mfg_last_cuda_error()
    s.close()


def test_static_norm_large_zero_and_no_allocation():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from minifs_b200 import _lib

    lib = _lib.load()
    stream = torch.cuda.current_stream()
    out = torch.full((5,), -1.0, dtype=torch.float64, device="cuda")

    def call(res, n):
        rc = lib.mfg_residual_norm_static(ct.c_void_p(res.data_ptr()), n,
                                          ct.c_void_p(out.data_ptr()),
                                          ct.c_void_p(stream.cuda_stream))
        assert rc == 0, lib.mfg_last_cuda_error()
        torch.cuda.synchronize()
        return out.cpu().numpy().copy()

    n = 6 * 64 ** 3
    rng = np.random.default_rng(11)
    host = rng.standard_normal((5, n)) * np.array([1e-3, 1e-1, 1e-2, 1e-2, 1e2])[:, None]
    res = torch.from_numpy(host.ravel()).to("cuda")
    expected = np.sqrt(np.sum(host * host, axis=1))
    for _ in range(2):
        np.testing.assert_allclose(call(res, n), expected, rtol=1e-12, atol=0)

    # no cells: the norms are zero
    np.testing.assert_array_equal(call(res, 0), np.zeros(5))

    # nothing is allocated on the device by further calls (the first calls
    # above have loaded the module and resolved the scratch address)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        call(res, n)
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
