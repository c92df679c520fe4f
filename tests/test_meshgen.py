"""Seeded mesh generator: counts, orientation, file round trip."""
import os
import tempfile

import numpy as np
import pytest

from minifs_b200 import meshgen


@pytest.mark.parametrize("n", [2, 5])
def test_counts_and_layout(n):
    m = meshgen.cube_mesh(n, jitter=0.15, seed=3)
    assert m.n_cell == 6 * n ** 3
    assert m.n_bface == 12 * n ** 2
    assert m.n_face == 12 * n ** 3 + 6 * n ** 2
    assert m.n_node == (n + 1) ** 3
    f2c = m.f2c.reshape(-1, 2)
    assert (f2c[:m.n_bface, 1] < 0).all() and (f2c[m.n_bface:, 1] >= 0).all()
    assert (f2c[m.n_bface:, 0] < f2c[m.n_bface:, 1]).all()
    cnt = np.bincount(f2c[:, 0], minlength=m.n_cell) + \
        np.bincount(f2c[m.n_bface:, 1], minlength=m.n_cell)
    assert (cnt == 4).all()


def test_normals_point_out_of_c1():
    m = meshgen.cube_mesh(4, jitter=0.2, seed=9)
    xyz = np.stack([m.x, m.y, m.z], 1)
    fn = m.f2n.reshape(-1, 3)
    p0, p1, p2 = xyz[fn[:, 0]], xyz[fn[:, 1]], xyz[fn[:, 2]]
    nrm = np.cross(p1 - p0, p2 - p0)
    f2c = m.f2c.reshape(-1, 2)
    cc = np.zeros((m.n_cell, 3))
    np.add.at(cc, f2c[:, 0], p0 + p1 + p2)
    np.add.at(cc, f2c[m.n_bface:, 1], (p0 + p1 + p2)[m.n_bface:])
    cc /= 12.0
    fc = (p0 + p1 + p2) / 3.0
    assert (np.einsum("ij,ij->i", nrm, fc - cc[f2c[:, 0]]) > 0).all()


def test_seeded_and_reproducible():
    a = meshgen.cube_mesh(3, jitter=0.15, seed=1)
    b = meshgen.cube_mesh(3, jitter=0.15, seed=1)
    c = meshgen.cube_mesh(3, jitter=0.15, seed=2)
    assert np.array_equal(a.x, b.x) and not np.array_equal(a.x, c.x)


def test_mfl_round_trip():
    m = meshgen.channel_mesh(6, 2, 2)
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "g.mfl")
        meshgen.write_mfl(m, p)
        r = meshgen.read_mfl(p)
        assert np.array_equal(r.x, m.x) and np.array_equal(r.f2n, m.f2n)
        assert np.array_equal(r.f2c, m.f2c) and r.n_bface == m.n_bface
        assert os.path.getsize(p) == 12 + 24 * m.n_node + 4 * m.n_face + 4 * m.f2n.size + \
            8 * m.n_face + 8
