"""The persistent sweeps' chunk assignment, planned on the host through
mfg_plan_chunks (no GPU): every cell in a chunk, the vote's even spread of
each level, the transverse grids' labels monotone along every dependency
(so that a dependency path crosses at most Pa + Pb - 2 chunk boundaries),
the model's own choice, and the checks of the tables."""
import ctypes as ct

import numpy as np
import pytest

from minifs_b200 import _lib, grid as gr, meshgen

VOTE, T_XY, T_XZ, T_YZ, T_ANY = 0, 1, 2, 3, 4


def sweep_tables(n=10, fwd=True):
    """A jittered cube's LU-SGS sweep in cell order: a cell depends on its
    face neighbours earlier in the sweep (lower ids forward, higher ids
    backward); levels by longest dependency path; cells sorted by (level,
    id); the dependency lists by position, ghosts (ids >= C) included."""
    mesh = meshgen.cube_mesh(n, jitter=0.15, seed=5)
    p = gr.make_params(mach=0.5, alpha=2.0, cfl_start=10.0)
    pg = gr.prepare(mesh, p)
    C = pg.n_cell
    f2c = np.asarray(pg.arrays["f2c"]).reshape(-1, 2)
    nbrs = [[] for _ in range(C)]
    for a, b in f2c:
        if a < C:
            nbrs[a].append(int(b))
        if b < C:
            nbrs[b].append(int(a))
    level = np.zeros(C, np.int64)
    ids = range(C) if fwd else range(C - 1, -1, -1)
    for c in ids:
        deps = [d for d in nbrs[c] if d < C and (d < c if fwd else d > c)]
        level[c] = 1 + max(level[d] for d in deps) if deps else 0
    cells = np.lexsort((np.arange(C), level)).astype(np.int32)
    L = int(level.max()) + 1
    lptr = np.searchsorted(level[cells], np.arange(L + 1)).astype(np.int32)
    lists = [[d for d in nbrs[c] if d >= C or (d < c if fwd else d > c)] for c in cells]
    sptr = np.zeros(C + 1, np.int32)
    sptr[1:] = np.cumsum([len(x) for x in lists])
    nbs = np.array([d for x in lists for d in x], np.int32)
    xyz = [np.ascontiguousarray(pg.arrays[k][:C]) for k in ("xcc", "ycc", "zcc")]
    return C, L, lptr, cells, sptr, nbs, xyz


def plan(t, P, G, force, geo=True, **over):
    C, L, lptr, cells, sptr, nbs, xyz = t
    args = dict(C=C, L=L, lptr=lptr, cells=cells, sptr=sptr, nbs=nbs)
    args.update(over)
    assign = np.full(max(C, 1), -7, np.int32)
    grid = np.zeros(2, np.int32)
    est = np.zeros(1)
    lib = _lib.load()
    null = ct.POINTER(ct.c_double)()
    rc = lib.mfg_plan_chunks(args["C"], args["L"], _lib.ptr(args["lptr"], _lib.i32p),
                             _lib.ptr(args["cells"], _lib.i32p), _lib.ptr(args["sptr"], _lib.i32p),
                             _lib.ptr(args["nbs"], _lib.i32p),
                             *([_lib.ptr(a) for a in xyz] if geo else [null] * 3),
                             P, G, force, _lib.ptr(assign, _lib.i32p), _lib.ptr(grid, _lib.i32p),
                             _lib.ptr(est))
    return rc, assign[:C], tuple(int(x) for x in grid), float(est[0])


def dependencies(t):
    C, L, lptr, cells, sptr, nbs, xyz = t
    for i, c in enumerate(cells):
        for d in nbs[sptr[i]:sptr[i + 1]]:
            if d < C:
                yield int(c), int(d)


@pytest.fixture(scope="module", params=[True, False], ids=["forward", "backward"])
def tables(request):
    return sweep_tables(10, fwd=request.param)


def test_vote_spreads_every_level(tables):
    C, L, lptr, cells = tables[:4]
    P = 12
    rc, a, grid, est = plan(tables, P, 16, VOTE)
    assert rc == VOTE and grid == (0, 0) and est > 0
    assert a.min() >= 0 and a.max() < P
    for l in range(L):
        lv = a[cells[lptr[l]:lptr[l + 1]]]
        quota = -(-(lptr[l + 1] - lptr[l]) // P)
        assert np.bincount(lv, minlength=P).max() <= quota, l


@pytest.mark.parametrize("force", [T_XY, T_XZ, T_YZ])
def test_transverse_labels_monotone_along_dependencies(tables, force):
    P = 12
    rc, a, (pa, pb), est = plan(tables, P, 16, force)
    assert rc == force and pa >= 1 and pb >= 1 and pa * pb <= P and est > 0
    la, lb = a % pa, a // pa
    assert a.min() >= 0 and lb.max() < pb
    # per axis one direction for every dependency (the maximum or the minimum)
    for lab in (la, lb):
        steps = np.array([np.sign(lab[c] - lab[d]) for c, d in dependencies(tables)])
        assert (steps >= 0).all() or (steps <= 0).all()
    # hence a chain of dependencies changes chunk at most Pa + Pb - 2 times:
    # follow the longest one back from the last level
    C, L, lptr, cells, sptr, nbs, _ = tables
    pos = np.empty(C, np.int64)
    pos[cells] = np.arange(C)
    level = np.searchsorted(lptr, pos, side="right") - 1
    c, crossings = int(cells[-1]), 0
    while True:
        ds = [int(d) for d in nbs[sptr[pos[c]]:sptr[pos[c] + 1]] if d < C]
        if not ds:
            break
        d = max(ds, key=lambda x: level[x])
        crossings += a[d] != a[c]
        c = d
    assert crossings <= pa + pb - 2


def test_model_choice_and_determinism(tables):
    r1 = plan(tables, 12, 16, -1)
    r2 = plan(tables, 12, 16, -1)
    assert r1[0] in (VOTE, T_XY, T_XZ, T_YZ)
    np.testing.assert_array_equal(r1[1], r2[1])
    assert r1[2] == r2[2] and r1[3] == r2[3]
    # the best transverse grid is one of the three pairs' grids
    rc, a, grid, est = plan(tables, 12, 16, T_ANY)
    assert rc in (T_XY, T_XZ, T_YZ) and grid[0] * grid[1] <= 12
    # without centroids a forced transverse assignment falls back to the vote
    rc, a, grid, est = plan(tables, 12, 16, T_XY, geo=False)
    assert rc == VOTE and grid == (0, 0)


def test_inconsistent_tables_are_refused():
    t = sweep_tables(4)
    C, L, lptr, cells, sptr, nbs, xyz = t
    bad_l = lptr.copy()
    bad_l[-1] -= 1
    assert plan(t, 4, 16, -1, lptr=bad_l)[0] == -1
    bad_c = cells.copy()
    bad_c[1] = bad_c[0]
    assert plan(t, 4, 16, -1, cells=bad_c)[0] == -1
    bad_n = nbs.copy()
    bad_n[0] = -3
    assert plan(t, 4, 16, -1, nbs=bad_n)[0] == -1
    assert plan(t, 0, 16, -1)[0] == -1
    assert plan(t, 4, 16, 9)[0] == -1
