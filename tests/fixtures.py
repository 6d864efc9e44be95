"""Helpers shared by the tests: load a golden fixture back into an SW2Case."""
import os

import numpy as np

from adh_kraken_b200.mesh import SW2Case

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    z = np.load(os.path.join(GOLDEN, name))
    series = {}
    for k in (0, 1, 2):
        if f"series{k}_t" in z:
            series[k] = (z[f"series{k}_t"], z[f"series{k}_v"])
    case = SW2Case(name, z["xyz"], z["tri"], z["seg"], z["seg_kind"], z["sol0"], float(z["dt"]), int(z["nsteps"]),
                   series, t0=float(z["t0"]))
    return case, z


def rel_err(a, b):
    """max |a-b| / max |b| per variable (h, u, v) of a node-major state"""
    out = []
    for k in range(3):
        x, y = a[k::3], b[k::3]
        out.append(float(np.abs(x - y).max() / max(np.abs(y).max(), 1e-300)))
    return out
