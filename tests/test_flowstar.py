"""FlowStar grid and bc.para files through the library's C reader and
writer (mfg_mfl_*, mfg_bc_*): the byte layout the reference reads (golden
file hashes), its face flip and boundary count, partitioned files'
interface block, and the errors for damaged files.  Host only."""
import hashlib

import numpy as np
import pytest

from helpers import GOLDEN_CASES, load_golden, raw_mesh_from_golden
from minifs_b200 import _lib, flowstar, grid as gr, meshgen


def _same_mesh(a, b):
    assert (a.n_node, a.n_face, a.n_cell, a.n_bface) == (b.n_node, b.n_face, b.n_cell, b.n_bface)
    for k in ("x", "y", "z"):
        assert np.asarray(getattr(a, k)).tobytes() == \
            np.asarray(getattr(b, k), np.float64).tobytes(), k
    for k in ("nnpf", "f2n", "f2c"):
        assert np.array_equal(np.asarray(getattr(a, k)), np.asarray(getattr(b, k))), k


def _box():
    m = meshgen.box_mesh(5, 4, 3, jitter=0.2, seed=3, bc_types=(3, 6, 4, 4, 5, 6))
    m.patches = [(i + 1, t) for i, t in enumerate((3, 6, 4, 4, 5, 6))]
    return m


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_written_file_is_the_one_the_reference_read(name, tmp_path):
    """The C writer produces byte for byte the grid file of each golden case
    (its SHA-256 was taken from the file the reference ran on)."""
    d = load_golden(name)
    m = raw_mesh_from_golden(d)
    flowstar.write_grid(m, tmp_path / "g.mfl")
    assert hashlib.sha256((tmp_path / "g.mfl").read_bytes()).hexdigest() == \
        bytes(d["mfl_sha256"]).decode()


def test_read_matches_python_reader_and_writer_bytes(tmp_path):
    m = _box()
    p_py, p_c = tmp_path / "py.mfl", tmp_path / "c.mfl"
    meshgen.write_mfl(m, str(p_py))
    flowstar.write_grid(m, p_c)
    assert p_py.read_bytes() == p_c.read_bytes()
    got, itf = flowstar.read_grid(p_c)
    _same_mesh(got, meshgen.read_mfl(str(p_py)))
    _same_mesh(got, m)
    assert len(itf.nbz) == 0 and len(itf.nbsn) == 0


def test_boundary_on_the_left_is_flipped(tmp_path):
    """A face stored with its boundary first reads back as the reference
    leaves it: cells swapped, nodes after the first reversed."""
    m = _box()
    stored = meshgen.RawMesh(x=m.x, y=m.y, z=m.z, nnpf=m.nnpf.copy(), f2n=m.f2n.copy(),
                             f2c=m.f2c.copy(), n_cell=m.n_cell, n_bface=m.n_bface)
    for i in (0, 3, m.n_bface - 1):
        stored.f2c[2 * i], stored.f2c[2 * i + 1] = stored.f2c[2 * i + 1], stored.f2c[2 * i]
        s = 3 * i
        stored.f2n[s + 1], stored.f2n[s + 2] = stored.f2n[s + 2], stored.f2n[s + 1]
    flowstar.write_grid(stored, tmp_path / "g.mfl")
    got, _ = flowstar.read_grid(tmp_path / "g.mfl")
    _same_mesh(got, m)
    assert got.n_bface == m.n_bface


def test_interface_block_round_trip(tmp_path):
    m = _box()
    itf = flowstar.Interfaces(nbz=np.array([1, 2, 2], np.int32),
                              nbf=np.array([7, 0, 11], np.int32),
                              nbsn=np.array([3, 4], np.int32), nbzn=np.array([1, 2], np.int32),
                              nbrn=np.array([30, 40], np.int32))
    flowstar.write_grid(m, tmp_path / "p.mfl", itf)
    got, gi = flowstar.read_grid(tmp_path / "p.mfl")
    _same_mesh(got, m)
    for k in ("nbz", "nbf", "nbsn", "nbzn", "nbrn"):
        assert np.array_equal(getattr(gi, k), getattr(itf, k)), k


def test_file_without_interface_block_reads_as_serial(tmp_path):
    m = _box()
    flowstar.write_grid(m, tmp_path / "g.mfl")
    raw = (tmp_path / "g.mfl").read_bytes()
    (tmp_path / "short.mfl").write_bytes(raw[:-8])  # drop n_iface = n_inode = 0
    got, itf = flowstar.read_grid(tmp_path / "short.mfl")
    _same_mesh(got, m)
    assert len(itf.nbz) == 0


def _code(fn, *a):
    with pytest.raises(_lib.MfgError) as e:
        fn(*a)
    return e.value.code


def test_damaged_grid_files_are_io_errors(tmp_path):
    m = _box()
    flowstar.write_grid(m, tmp_path / "g.mfl")
    raw = (tmp_path / "g.mfl").read_bytes()
    N, F = m.n_node, m.n_face
    cuts = [0, 8, 12 + 24 * N - 4, 12 + 24 * N + 4 * F + 4, len(raw) - 12, len(raw) - 6]
    for k, cut in enumerate(cuts):
        p = tmp_path / f"cut{k}.mfl"
        p.write_bytes(raw[:cut])
        assert _code(flowstar.read_grid, p) == -9, cut
    (tmp_path / "tail.mfl").write_bytes(raw + b"\x00\x00\x00\x00")
    assert _code(flowstar.read_grid, tmp_path / "tail.mfl") == -9
    bad = bytearray(raw)
    bad[4:8] = np.array([-5], np.int32).tobytes()  # negative face count
    (tmp_path / "neg.mfl").write_bytes(bytes(bad))
    assert _code(flowstar.read_grid, tmp_path / "neg.mfl") == -9
    bad = bytearray(raw)
    off = 12 + 24 * N
    bad[off:off + 4] = np.array([0], np.int32).tobytes()  # a face with no nodes
    (tmp_path / "zero.mfl").write_bytes(bytes(bad))
    assert _code(flowstar.read_grid, tmp_path / "zero.mfl") == -9
    bad = bytearray(raw)
    bad[off:off + 4] = np.array([1 << 30], np.int32).tobytes()  # more nodes than the file holds
    (tmp_path / "huge.mfl").write_bytes(bytes(bad))
    assert _code(flowstar.read_grid, tmp_path / "huge.mfl") == -9
    assert _code(flowstar.read_grid, tmp_path / "missing.mfl") == -9


def test_bc_file_round_trip_and_errors(tmp_path):
    patches = [(1, 3), (2, 6), (3, 4), (7, 61), (5, 10)]
    flowstar.write_bc(patches, tmp_path / "bc.para")
    assert (tmp_path / "bc.para").read_text() == "5\n1 3\n2 6\n3 4\n7 61\n5 10\n"
    assert flowstar.read_bc(tmp_path / "bc.para") == patches
    m = _box()
    meshgen.write_bc(m, str(tmp_path / "py.para"))
    assert flowstar.read_bc(tmp_path / "py.para") == m.patches
    assert _code(flowstar.read_bc, tmp_path / "bc.para", 4) == -1  # more records than room
    (tmp_path / "short.para").write_text("3\n1 3\n2\n")
    assert _code(flowstar.read_bc, tmp_path / "short.para") == -9
    (tmp_path / "text.para").write_text("two\n")
    assert _code(flowstar.read_bc, tmp_path / "text.para") == -9
    assert _code(flowstar.read_bc, tmp_path / "none.para") == -9


def test_case_from_files_prepares_like_the_mesh(tmp_path):
    m = _box()
    flowstar.write_grid(m, tmp_path / "g.mfl")
    flowstar.write_bc(m.patches, tmp_path / "bc.para")
    got = flowstar.read_case(tmp_path / "g.mfl", tmp_path / "bc.para")
    p = gr.make_params(mach=0.5, alpha=2.0, cfl_start=10.0)
    a = gr.prepare(got, p)
    b = gr.prepare(m, p)
    for k in b.arrays:
        assert np.asarray(a.arrays[k]).tobytes() == np.asarray(b.arrays[k]).tobytes(), k
    assert a.q0.tobytes() == b.q0.tobytes()
