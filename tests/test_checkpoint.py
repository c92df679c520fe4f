"""Checkpoint files (mfg_checkpoint_write / mfg_checkpoint_read) on the CPU:
round trip and the errors of a damaged or foreign file."""
import ctypes as ct

import numpy as np
import pytest

from minifs_b200 import _lib


def _write(path, n_cell, n, it, mx, mn, q):
    lib = _lib.load()
    return lib.mfg_checkpoint_write(str(path).encode(), n_cell, n, it, mx, mn, _lib.ptr(q))


def _read(path, n_cell, n):
    lib = _lib.load()
    q = np.zeros(5 * n)
    it, mx, mn = ct.c_int32(-1), ct.c_double(), ct.c_double()
    rc = lib.mfg_checkpoint_read(str(path).encode(), n_cell, n, ct.byref(it), ct.byref(mx),
                                 ct.byref(mn), _lib.ptr(q))
    return rc, it.value, mx.value, mn.value, q


def test_round_trip(tmp_path):
    rng = np.random.default_rng(3)
    q = rng.standard_normal(5 * 70)
    p = tmp_path / "run.ckpt"
    assert _write(p, 60, 70, 123, 0.25, 1e-9, q) == 0
    rc, it, mx, mn, back = _read(p, 60, 70)
    assert rc == 0 and it == 123 and mx == 0.25 and mn == 1e-9
    assert np.array_equal(back, q)


def test_errors(tmp_path):
    q = np.ones(5 * 10)
    p = tmp_path / "a.ckpt"
    assert _write(p, 8, 10, 5, 1.0, 0.5, q) == 0
    assert _read(p, 8, 11)[0] == -1  # another grid
    assert _read(p, 9, 10)[0] == -1
    assert _read(tmp_path / "missing.ckpt", 8, 10)[0] == -9
    data = p.read_bytes()
    (tmp_path / "short.ckpt").write_bytes(data[:-8])
    assert _read(tmp_path / "short.ckpt", 8, 10)[0] == -9
    (tmp_path / "magic.ckpt").write_bytes(b"X" + data[1:])
    assert _read(tmp_path / "magic.ckpt", 8, 10)[0] == -9
    assert _write(p, 8, 7, 5, 1.0, 0.5, q) == -1  # n below n_cell
    assert _write(p, 8, 10, -1, 1.0, 0.5, q) == -1
