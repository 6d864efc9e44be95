"""Test infrastructure: talk to the compiled reference harness (oracle/_ref/).

``write_case`` writes a :class:`adh_kraken_b200.mesh.SW2Case` in the harness's
binary case format (read by ``read_case`` in oracle/ref_harness.c);
``read_records`` parses the harness's output; ``run_harness`` runs one mode.
Only tests, the smoke check, fixture generation and bench.py's CPU-baseline leg use
this module.
"""
from __future__ import annotations

import os
import struct
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
HARNESS = os.path.join(HERE, "_ref", "adh_ref_harness")
# the reference's objects with assemble_residual / assemble_jacobian taken from the
# product's reference-signature glue (GPU); runs only where a GPU is present
GLUE_HARNESS = os.path.join(HERE, "_ref", "adh_refglue_harness")


def harness_available(binary=HARNESS) -> bool:
    return os.path.exists(binary)


def write_case(case, path, sol=None, sol_old=None, sol_older=None):
    V = case.nnodes
    sol0 = case.sol0 if sol is None else sol
    so = case.sol0 if sol_old is None else sol_old
    soo = case.sol0 if sol_older is None else sol_older
    with open(path, "wb") as f:
        f.write(struct.pack("<ii", 0x43325753, 1))
        f.write(struct.pack("<5i", V, case.ntri, case.nseg, case.nsteps, case.max_nonlin_it))
        f.write(struct.pack("<5d", case.dt, case.t0, case.tol_nonlin, case.inc_nonlin, case.gravity))
        f.write(np.ascontiguousarray(case.xyz, dtype="<f8").tobytes())
        f.write(np.ascontiguousarray(case.tri, dtype="<i4").tobytes())
        f.write(np.ascontiguousarray(case.seg, dtype="<i4").tobytes())
        f.write(np.ascontiguousarray(case.seg_kind, dtype="<i4").tobytes())
        for a in (sol0, so, soo):
            f.write(np.ascontiguousarray(a, dtype="<f8").tobytes())
        f.write(struct.pack("<i", len(case.series)))
        for sid in sorted(case.series):
            t, v = case.series[sid]
            f.write(struct.pack("<ii", sid, len(t)))
            f.write(np.ascontiguousarray(t, dtype="<f8").tobytes())
            f.write(np.ascontiguousarray(v, dtype="<f8").tobytes())


def read_records(path):
    out = {}
    with open(path, "rb") as f:
        data = f.read()
    pos = 0
    while pos < len(data):
        name = data[pos:pos + 32].split(b"\0", 1)[0].decode()
        typ = chr(data[pos + 32])
        (count,) = struct.unpack_from("<q", data, pos + 33)
        pos += 41
        dt = np.dtype("<f8") if typ == "d" else np.dtype("<i4")
        out[name] = np.frombuffer(data, dtype=dt, count=count, offset=pos).copy()
        pos += count * dt.itemsize
    return out


class HarnessRun:
    """One harness run in the background (a subprocess): start() returns at once,
    wait() returns its records.  Used where the reference's CPU run overlaps other work."""

    def __init__(self, mode, case, extra=(), binary=HARNESS):
        if not harness_available(binary):
            raise RuntimeError(f"reference harness not built ({binary})")
        self.td = tempfile.TemporaryDirectory()
        cpath = os.path.join(self.td.name, "case.bin")
        self.opath = os.path.join(self.td.name, "out.bin")
        write_case(case, cpath)
        self.p = subprocess.Popen([binary, mode, cpath, self.opath, *map(str, extra)], stdout=subprocess.DEVNULL,
                                  stderr=subprocess.PIPE, cwd=self.td.name)

    def wait(self, timeout=3600):
        _, err = self.p.communicate(timeout=timeout)
        try:
            if self.p.returncode != 0:
                raise RuntimeError(f"harness failed ({self.p.returncode}): {err.decode()[-2000:]}")
            return read_records(self.opath)
        finally:
            self.td.cleanup()


def run_harness(mode, case=None, extra=(), sol=None, sol_old=None, sol_older=None, env=None, timeout=3600,
                in_path=None, binary=HARNESS):
    if not harness_available(binary):
        raise RuntimeError(f"reference harness not built ({binary})")
    with tempfile.TemporaryDirectory() as td:
        cpath = os.path.join(td, "case.bin")
        opath = os.path.join(td, "out.bin")
        if case is not None:
            write_case(case, cpath, sol, sol_old, sol_older)
        elif in_path is not None:         # a mode that reads a file of its own (geo)
            cpath = os.path.abspath(in_path)
        else:
            cpath = "-"
        e = dict(os.environ)
        if env:
            e.update(env)
        # cwd: the reference's grid reader writes a node listing file into the working directory
        r = subprocess.run([binary, mode, cpath, opath, *map(str, extra)], capture_output=True, env=e,
                           timeout=timeout, cwd=td)
        if r.returncode != 0:
            raise RuntimeError(f"harness {mode} failed ({r.returncode}): {r.stderr.decode()[-2000:]}")
        return read_records(opath)


def run_bcx(records):
    """Discharge / tailwater segment residuals computed by the reference's own boundary
    integrals and roughness law (harness mode ``bcx``) for records of 21 doubles
    {kind, nx, ny, djac, dt, g, h0, h1, u0, v0, u1, v1, z0, q_series, conveyance,
    rough_height, tail_elev, perturbation, perturb_node, perturb_var, perturb_sign}."""
    rec = np.ascontiguousarray(records, dtype="<f8").reshape(-1, 21)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "bcx.bin")
        with open(p, "wb") as f:
            f.write(struct.pack("<i", rec.shape[0]))
            f.write(rec.tobytes())
        out = run_harness("bcx", in_path=p)
    return out["seg_resid"].reshape(-1, 6)


def run_params_series(path):
    """The BC time series of a ``.params`` file as the reference's own reader builds them
    (harness mode ``params``): {id: (times, values)} in list order."""
    out = run_harness("params", in_path=path)
    ids, sizes = out["ids"], out["sizes"]
    res, e = {}, 0
    for sid, n in zip(ids.tolist(), sizes.tolist()):
        res[int(sid)] = (out["times"][e:e + n], out["values"][e:e + n])
        e += n
    return res
