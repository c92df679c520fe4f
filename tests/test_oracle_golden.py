"""The CPU oracle (oracle/minifs_oracle.c) against the golden fixtures made
by the reference itself (tests/golden/make_golden.py): bit-for-bit."""
import numpy as np
import pytest

from helpers import GOLDEN_CASES, assert_bitwise, golden_params, load_golden, oracle_from


def _oracle(d):
    return oracle_from(d, golden_params(d), d["init.q"], d["dims"])


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_oracle_matches_reference_every_routine(name):
    d = load_golden(name)
    o = _oracle(d)
    iters = d["meta"]["case"]["iters"]
    dumped = sorted(int(k[2:].split(".")[0]) for k in d if k.startswith("it") and k.endswith(".res"))
    assert dumped, "fixture has no per-iteration dumps"
    norms = []
    for it in range(iters):
        o.zero_residuals()
        o.inviscid_flux()
        if it in dumped:
            assert_bitwise(o.res, d[f"it{it}.res"], f"{name} it{it} res")
        o.compute_timestep()
        if it in dumped:
            assert_bitwise(o.dt, d[f"it{it}.dt"], f"{name} it{it} dt")
        o.forward_lusgs()
        if it in dumped:
            assert_bitwise(o.diag, d[f"it{it}.diag"], f"{name} it{it} diag")
            assert_bitwise(o.dq, d[f"it{it}.dq_lusgs"], f"{name} it{it} DQ")
            assert_bitwise(o.q, d[f"it{it}.q"], f"{name} it{it} q")
        o.calculate_gradient()
        if it in dumped:
            for ax in "xyz":
                assert_bitwise(getattr(o, "dqd" + ax), d[f"it{it}.dqd{ax}"], f"{name} it{it} dqd{ax}")
            assert tuple(o.dt_extrema) == tuple(d[f"it{it}.dt_extrema"])
        o.s.iter_done += 1
        norms.append(o.residual_norm())
    assert_bitwise(o.q, d["final.q"], f"{name} final q")
    assert_bitwise(o.res, d["final.res"], f"{name} final res")
    assert_bitwise(np.concatenate(norms), d["norms"], f"{name} norms")


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_oracle_initial_gradient(name):
    d = load_golden(name)
    o = _oracle(d)
    o.calculate_gradient()
    assert_bitwise(o.dqdx, d["init.dqdx"], "AllocAndCalQuantityGradient dqdx")


def test_oracle_on_tdtree_renumbered_grid():
    """Serial arithmetic on the reference's TDTree renumbering reproduces the
    TDTree build's state: its flux, time step and LU-SGS are the serial ones
    on the renumbered grid (only its unused gradient sums differently)."""
    d = load_golden("tdtree8")
    o = _oracle(d)
    norms = o.iterate(d["meta"]["case"]["iters"])
    assert_bitwise(o.q, d["final.q"], "serial-on-renumbered q")
    assert_bitwise(o.res, d["final.res"], "serial-on-renumbered res")
    assert_bitwise(o.dqdx, d["final.dqdx"], "serial-on-renumbered dqdx")
    assert_bitwise(norms.reshape(-1), d["norms"], "norms")
    assert_bitwise(d["tdtree.final.q"], d["final.q"], "TDTree build q == serial on renumbered")


def test_oracle_iterate_equals_stepwise():
    d = load_golden("cube4")
    a = _oracle(d)
    b = _oracle(d)
    na = a.iterate(5)
    for _ in range(5):
        b.step()
    assert_bitwise(a.q, b.q, "iterate vs step")
    assert_bitwise(na[-1], b.residual_norm(), "norm")
