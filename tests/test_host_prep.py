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
