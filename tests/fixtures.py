"""Helpers shared by the tests: load a golden fixture back into an SW2Case."""
import os

import numpy as np

from adh_kraken_b200.mesh import SW2Case

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def reference_src():
    """The reference tree's src/ directory as oracle/Makefile recorded it when it
    compiled the reference (oracle/_ref/ref_src_path.txt), or None where that tree is
    not on this machine (the tests that read it then skip)."""
    rec = os.path.join(ROOT, "oracle", "_ref", "ref_src_path.txt")
    if not os.path.exists(rec):
        return None
    path = open(rec).read().strip()
    return path if os.path.exists(os.path.join(path, "include", "adh.h")) else None


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
