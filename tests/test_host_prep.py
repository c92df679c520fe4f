"""The product's host preprocessing (C++ restatement of SpecifyBC,
ComputeMetrics, AllocAndInitFlowfield + SetGhostVariables,
ComputeWeight3D_Node, FindNodeSYMM and the parameter derivation) against the
reference's own outputs: bit-for-bit."""
import hashlib
import os
import tempfile

import numpy as np
import pytest

from helpers import (GOLDEN_CASES, PARAM_NAMES, assert_bitwise, load_golden,
                     make_product_params, prepare_product, raw_mesh_from_golden)
from minifs_b200 import meshgen

PREP = ["f2c", "bctype", "xfn", "yfn", "zfn", "area", "xfc", "yfc", "zfc", "xcc", "ycc", "zcc",
        "vol", "wnode", "nmark", "wbface", "nodesymm", "xfn_n_symm", "yfn_n_symm", "zfn_n_symm"]


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_generator_reproduces_reference_input(name):
    d = load_golden(name)
    m = raw_mesh_from_golden(d)
    with tempfile.TemporaryDirectory() as t:
        p = os.path.join(t, "g.mfl")
        meshgen.write_mfl(m, p)
        with open(p, "rb") as f:
            sha = hashlib.sha256(f.read()).hexdigest()
    assert sha == bytes(d["mfl_sha256"]).decode()


@pytest.mark.parametrize("name", GOLDEN_CASES + ("tdtree8",))
def test_params_derivation(name):
    d = load_golden(name)
    p = make_product_params(d).as_dict()
    for k, v in zip(PARAM_NAMES, d["params"]):
        if k in p:
            assert p[k] == v, k


@pytest.mark.parametrize("name", GOLDEN_CASES + ("tdtree8",))
def test_preprocessing_bitexact(name):
    d = load_golden(name)
    pg, _ = prepare_product(d)
    for k in PREP:
        assert_bitwise(pg.arrays[k], d[k], f"{name} {k}")
    assert_bitwise(pg.q0, d["init.q"], f"{name} initial state incl. ghosts")

    def cmap(nnpc, c2n, w):
        cells = np.repeat(np.arange(len(nnpc)), nnpc)
        return dict(zip(zip(cells.tolist(), c2n.tolist()), w.tolist()))

    assert cmap(pg.arrays["nnpc"], pg.arrays["c2n"], pg.arrays["wc2n"]) == \
        cmap(d["nnpc"], d["c2n"], d["wc2n"])


def test_bad_volume_is_reported():
    """An inverted cell makes CellVolCentroid fail (the reference exits)."""
    from minifs_b200 import _lib, grid as gr
    m = meshgen.cube_mesh(2, jitter=0.0)
    # swap two nodes of an interior face to break orientation of its c1
    g = m.n_bface
    m.f2n[3 * g + 1], m.f2n[3 * g + 2] = m.f2n[3 * g + 2], m.f2n[3 * g + 1]
    m.x = m.x.copy()
    # collapse a cell: move an interior node far outside
    p = gr.make_params(mach=0.5, alpha=2.0, cfl_start=10.0)
    m.x[13] = 5.0
    with pytest.raises(_lib.MfgError) as e:
        gr.prepare(m, p)
    assert e.value.code == -7


def test_state_rel_err_scales():
    """The FP64/mixed comparison measures velocity against the speed and the
    gauge pressure against the absolute pressure."""
    import numpy as np
    from minifs_b200.compare import state_rel_err
    n = 4
    b = np.concatenate([np.full(n, 1.2), np.full(n, 1.0), np.zeros(n), np.full(n, 0.02),
                        np.zeros(n)])
    a = b.copy()
    a[2 * n] = 1e-6           # v: 1e-6 against a speed of ~1
    a[4 * n + 1] = 2e-6       # gauge p: 2e-6 against p + p_bar = 2
    e = state_rel_err(a, b, n, 2.0)
    # velocity 1e-6 / |(1, 0, 0.02)|, pressure 2e-6 / 2: the larger
    assert abs(e["max_norm"] - max(1e-6 / np.hypot(1.0, 0.02), 1e-6)) < 1e-15
    assert e["l2"] < 1e-6 and e["l2"] > 0
    assert state_rel_err(b, b, n, 2.0) == {"l2": 0.0, "max_norm": 0.0}
