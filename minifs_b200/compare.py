"""Comparison of flow states between the FP64 and the mixed-precision forms."""
from __future__ import annotations

import numpy as np


def state_rel_err(a, b, n, p_bar):
    """Error of state a against state b (SoA rho, u, v, w, p over n cells and
    ghosts) on physical scales: density against density, the velocity vector
    against the speed, the gauge pressure against the absolute pressure
    p + p_bar.  (v and the gauge p are near zero in these flows, so their
    own magnitudes are no scale.)  Largest over the three, in the L2 and the
    max norm."""
    blk = [a[k * n:(k + 1) * n] - b[k * n:(k + 1) * n] for k in range(5)]
    ref = [b[k * n:(k + 1) * n] for k in range(5)]
    vel_d = np.sqrt(blk[1] ** 2 + blk[2] ** 2 + blk[3] ** 2)
    vel = np.sqrt(ref[1] ** 2 + ref[2] ** 2 + ref[3] ** 2)
    pairs = [(blk[0], ref[0]), (vel_d, vel), (blk[4], ref[4] + p_bar)]
    l2 = max(float(np.linalg.norm(d) / np.linalg.norm(r)) for d, r in pairs)
    mx = max(float(np.max(np.abs(d)) / np.max(np.abs(r))) for d, r in pairs)
    return {"l2": l2, "max_norm": mx}


def state_component_err(a, b, n):
    """Error of state a against state b per component (rho, u, v, w, gauge
    p), each against its own magnitude: ||a_k - b_k||_2 / ||b_k||_2 and
    max|a_k - b_k| / max|b_k|.  Components near zero in a flow (v, the gauge
    pressure) read large here; state_rel_err gives their physical scale."""
    names = ("rho", "u", "v", "w", "p_gauge")
    out = {}
    for k, name in enumerate(names):
        d = a[k * n:(k + 1) * n] - b[k * n:(k + 1) * n]
        r = b[k * n:(k + 1) * n]
        nr, mr = float(np.linalg.norm(r)), float(np.max(np.abs(r)))
        out[name] = {"l2": float(np.linalg.norm(d)) / nr if nr > 0 else float(np.linalg.norm(d)),
                     "max": float(np.max(np.abs(d))) / mr if mr > 0 else float(np.max(np.abs(d)))}
    return out
