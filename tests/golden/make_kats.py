"""Regenerate tests/golden/kats.npz: known answers of single reference
functions on inputs chosen to reach each of their branches.

Runs ``oracle/_ref/minifs_kat`` (oracle/kat_harness.cpp linked with the
unmodified MiniFS sources, built by ``make -C oracle ref``), which calls
``RoeFlux_noprec`` (cal_flux.cpp:301-834) on a chunk of faces and
``FluxLUSGS3D`` (forward_lusgs.cpp:1271-1324) case by case and
``UpdateFlowField3D_CFL3d`` (forward_lusgs.cpp:1335-1488) on a grid of
loose cells, and stores the inputs with the reference's outputs.  Usage:  python tests/golden/make_kats.py

Face groups of the Roe cases (each with random unit normals unless noted):
  random      subsonic states with moderate jumps
  stagnation  velocities of 1e-3 of the sound speed: |vn| below the entropy
              fix's threshold 2*eps, so the fix replaces the first eigenvalue
  sonic       normal velocity within 1e-3 of the sound speed, either sign:
              the fix replaces |vn + c| or |vn - c|
  supersonic  |vn| of 2-3 sound speeds, either sign: no eigenvalue is fixed
  jump        density ratio up to 5, pressure ratio up to 10 across the face
  equal       identical states on both sides
  axis        normals along +-x, +-y, +-z (zero components)
Cell groups of the update cases: small increments, density drops and
pressure drops beyond 20% (the relaxation branches), both at once, and
increments past rho_max and p_max (the clamps).
Two parameter sets: Mach 0.5 with the reference's epsa_r = 0.1, and Mach
0.8395 with epsa_r = 0 (no entropy fix at all).
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
KAT = os.path.join(ROOT, "oracle", "_ref", "minifs_kat")

GROUPS = ("random", "stagnation", "sonic", "supersonic", "jump", "equal", "axis")
PER_GROUP = 100


def unit(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def roe_inputs(rng, p):
    """ql, qr [5][F] primitive states (rho, u, v, w, p - p_bar) and normals."""
    ql, qr, nrm, grp = [], [], [], []
    for g, name in enumerate(GROUPS):
        n = PER_GROUP
        nh = unit(rng, n)
        if name == "axis":
            ax = np.zeros((n, 3))
            ax[np.arange(n), np.arange(n) % 3] = np.where(np.arange(n) % 2, 1.0, -1.0)
            nh = ax
        rho_l = p.rho_s * rng.uniform(0.5, 2.0, n)
        pa_l = p.p_bar * rng.uniform(0.5, 2.0, n)
        a_l = np.sqrt(p.gam * pa_l / rho_l)
        if name == "stagnation":
            v_l = 1e-3 * a_l[:, None] * rng.uniform(-1, 1, (n, 3))
            rel = 1e-3
        elif name == "sonic":
            sign = np.where(rng.uniform(size=n) < 0.5, -1.0, 1.0)
            v_l = (sign * a_l * (1 + 1e-3 * rng.uniform(-1, 1, n)))[:, None] * nh
            rel = 1e-4
        elif name == "supersonic":
            sign = np.where(rng.uniform(size=n) < 0.5, -1.0, 1.0)
            v_l = (sign * a_l * rng.uniform(2, 3, n))[:, None] * nh
            rel = 0.05
        else:
            v_l = 0.8 * p.ainf * rng.uniform(-1, 1, (n, 3))
            rel = 0.1
        if name == "jump":
            rho_r = rho_l * rng.uniform(1.0, 5.0, n) ** np.where(rng.uniform(size=n) < 0.5, -1, 1)
            pa_r = pa_l * rng.uniform(1.0, 10.0, n) ** np.where(rng.uniform(size=n) < 0.5, -1, 1)
            v_r = 0.8 * p.ainf * rng.uniform(-1, 1, (n, 3))
        elif name == "equal":
            rho_r, pa_r, v_r = rho_l.copy(), pa_l.copy(), v_l.copy()
        else:
            rho_r = rho_l * (1 + rel * rng.uniform(-1, 1, n))
            pa_r = pa_l * (1 + rel * rng.uniform(-1, 1, n))
            scale = np.linalg.norm(v_l, axis=1, keepdims=True) + 1e-3 * a_l[:, None]
            v_r = v_l + rel * scale * rng.uniform(-1, 1, (n, 3))
        ql.append(np.vstack([rho_l, v_l.T, pa_l - p.p_bar]))
        qr.append(np.vstack([rho_r, v_r.T, pa_r - p.p_bar]))
        nrm.append(nh)
        grp.append(np.full(n, g, np.int32))
    ql, qr, nrm = np.hstack(ql), np.hstack(qr), np.vstack(nrm)
    area = 10.0 ** rng.uniform(-4, 0, ql.shape[1])
    return ql, qr, nrm, area, np.concatenate(grp)


def lusgs_inputs(rng, p, n=600):
    """Per case q[5] (primitive), dq[5] (conservative increment), n[3]."""
    rho = p.rho_s * rng.uniform(0.5, 2.0, n)
    pa = p.p_bar * rng.uniform(0.5, 2.0, n)
    vel = p.ainf * rng.uniform(-1, 1, (n, 3)) * rng.choice([0.001, 0.8, 2.5], n)[:, None]
    q = np.column_stack([rho, vel, pa - p.p_bar])
    e = pa / (p.gam - 1) + 0.5 * rho * (vel ** 2).sum(1)
    cons = np.column_stack([rho, rho[:, None] * vel, e])
    mag = rng.choice([0.0, 1e-6, 1e-3, 0.1], n)  # zero increments in a quarter of the cases
    dq = cons * mag[:, None] * rng.uniform(-1, 1, (n, 5))
    nh = unit(rng, n)
    nh[: n // 10] = np.eye(3)[np.arange(n // 10) % 3]
    return np.column_stack([q, dq, nh])


UPDATE_GROUPS = ("small", "rho_drop", "p_drop", "both_drop", "rho_high", "p_high")


def update_inputs(rng, p, per=100):
    """q [5][C] primitive states and DQ [5][C] conservative increments."""
    G = len(UPDATE_GROUPS)
    C = per * G
    grp = np.repeat(np.arange(G, dtype=np.int32), per)
    rho = p.rho_s * rng.uniform(0.5, 2.0, C)
    pa = p.p_bar * rng.uniform(0.5, 2.0, C)
    vel = 0.8 * p.ainf * rng.uniform(-1, 1, (C, 3))
    e = pa / (p.gam - 1) + 0.5 * rho * (vel ** 2).sum(1)
    cons = np.column_stack([rho, rho[:, None] * vel, e])
    dq = cons * 1e-3 * rng.uniform(-1, 1, (C, 5))
    drop = rng.uniform(0.25, 0.95, C)
    for g, name in enumerate(UPDATE_GROUPS):
        s = grp == g
        if name in ("rho_drop", "both_drop"):
            dq[s, 0] = -drop[s] * rho[s]
        if name in ("p_drop", "both_drop"):
            dq[s, 4] = -drop[s] * pa[s] / (p.gam - 1)
        if name == "rho_high":
            dq[s, 0] = (p.rho_max / rho[s]) * rng.uniform(1.5, 3.0, s.sum()) * rho[s]
        if name == "p_high":
            dq[s, 4] = (p.p_max + p.p_bar) * rng.uniform(1.5, 3.0, s.sum()) / (p.gam - 1)
    q = np.vstack([rho, vel.T, pa - p.p_bar])
    return q, np.ascontiguousarray(dq.T), grp


def run(mode, head, body):
    with tempfile.TemporaryDirectory() as d:
        fin, fout = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
        np.concatenate([np.asarray(head, np.float64), body.ravel()]).tofile(fin)
        subprocess.run([KAT, mode, fin, fout], check=True, stdout=subprocess.DEVNULL)
        return np.fromfile(fout, np.float64)


def main():
    from minifs_b200 import grid as gr
    if not os.path.exists(KAT):
        sys.exit("build the reference first: make -C oracle ref")
    out = {}
    for s, (mach, epsa_r, lhs) in enumerate(((0.5, 0.1, 1.0), (0.8395, 0.0, 1.5))):
        p = gr.make_params(mach=mach, alpha=2.0, epsa_r=epsa_r, lhs_omga=lhs)
        rng = np.random.default_rng(20260 + s)
        ql, qr, nrm, area, grp = roe_inputs(rng, p)
        F = ql.shape[1]
        body = np.concatenate([ql.ravel(), qr.ravel(), nrm[:, 0], nrm[:, 1], nrm[:, 2], area])
        flux = run("roe", [F, p.gam, p.p_bar, epsa_r], body).reshape(5, F)
        cases = lusgs_inputs(rng, p)
        lflux = run("lusgs", [len(cases), p.gam, p.p_bar, lhs], cases).reshape(-1, 5)
        uq, udq, ugrp = update_inputs(rng, p)
        C = uq.shape[1]
        lim = [p.rho_s, p.rho_min, p.rho_max, p.p_min, p.p_max]
        uq_out = run("update", [C, p.gam, p.p_bar, 0.0],
                     np.concatenate([lim, uq.ravel(), udq.ravel()])).reshape(5, C)
        out.update({f"s{s}_update_q": uq, f"s{s}_update_dq": udq, f"s{s}_update_group": ugrp,
                    f"s{s}_update_limits": np.array(lim), f"s{s}_update_out": uq_out})
        out.update({f"s{s}_params": np.array([mach, epsa_r, lhs, p.gam, p.p_bar]),
                    f"s{s}_ql": ql, f"s{s}_qr": qr, f"s{s}_normal": nrm, f"s{s}_area": area,
                    f"s{s}_group": grp, f"s{s}_roe_flux": flux,
                    f"s{s}_lusgs_in": cases, f"s{s}_lusgs_flux": lflux})
    np.savez_compressed(os.path.join(HERE, "kats.npz"), **out)
    print("wrote", os.path.join(HERE, "kats.npz"))


if __name__ == "__main__":
    main()
