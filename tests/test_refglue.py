"""The reference-signature glue (adh_kraken_b200/refglue/sw2_refglue.c) inside the
reference's own code.

oracle/Makefile links the reference's objects -- without src/residual/assemble_residual.c
and src/jacobian/assemble_jacobian.c -- with the glue and the CUDA library into
oracle/_ref/adh_refglue_harness.  There the reference's fe_newton calls the glue's
assemble_residual(SMODEL_SUPER*, SGRID*) / assemble_jacobian(SMODEL_SUPER*), which run on
the GPU, and mode "loop_gpu" installs fe_newton_gpu in adh_time_stepper[FE_NEWTON] under
the reference's time_loop (src/timeloop/time_loop.c:14-89).  Both are compared with the
unmodified reference running the same time_loop (oracle/_ref/adh_ref_harness "loop")."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from adh_kraken_b200.mesh import flume_case, small_delaunay_case
from fixtures import ROOT, reference_src, rel_err
from oracle.refio import GLUE_HARNESS, HARNESS, harness_available, run_harness

GLUE = os.path.join(ROOT, "adh_kraken_b200", "refglue")
needs_glue = pytest.mark.skipif(not (harness_available(HARNESS) and harness_available(GLUE_HARNESS)),
                                reason="reference harness or glue harness not built (oracle/_ref)")


@pytest.mark.skipif(reference_src() is None or shutil.which("gcc") is None, reason="reference tree or gcc absent")
def test_glue_compiles_against_the_reference_headers():
    src = reference_src()
    incs = ["-I", os.path.join(ROOT, "oracle", "shim"), "-I", os.path.join(ROOT, "include"), "-I", GLUE]
    for d, _, _ in os.walk(src):
        if "/test" not in d:
            incs += ["-I", d]
    r = subprocess.run(["gcc", "-std=gnu99", "-fcommon", "-fsyntax-only", "-Werror=implicit-function-declaration",
                        "-Werror=incompatible-pointer-types", "-Werror=int-conversion", "-Werror=return-type", *incs,
                        "-I", os.path.join(src, "test"), os.path.join(GLUE, "sw2_refglue.c")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]


@needs_glue
def test_glue_harness_replaces_the_reference_assembly():
    """The glue binary takes assemble_residual / assemble_jacobian from the glue (the
    reference's objects for them are left out) and the reference's fe_newton and time_loop
    from the reference."""
    nm = shutil.which("nm")
    if nm is None:
        pytest.skip("nm absent")
    out = subprocess.run([nm, GLUE_HARNESS], capture_output=True, text=True).stdout
    defined = {ln.split()[-1] for ln in out.splitlines() if len(ln.split()) == 3 and ln.split()[1] in "Tt"}
    for sym in ("assemble_residual", "assemble_jacobian", "fe_newton_gpu", "fe_newton", "time_loop"):
        assert sym in defined, sym
    for sym in ("load_elem_mat", "perturb_var", "load_global_resid"):   # only in the replaced reference files
        assert sym not in defined, sym


def _cases():
    return [flume_case(nsteps=100), small_delaunay_case(n=12, seed=5, nsteps=4)]


@pytest.mark.gpu
@needs_glue
@pytest.mark.parametrize("ci", [0, 1], ids=["flume101x11_100steps", "wetdry12_4steps"])
def test_reference_newton_on_gpu_assembly_is_bit_exact(ci):
    """The reference's own fe_newton and time_loop with the GPU assembly linked in: every
    step's state, success flag and Newton count equal the unmodified reference's."""
    case = _cases()[ci]
    ref = run_harness("loop", case)
    glue = run_harness("loop", case, binary=GLUE_HARNESS)
    assert np.array_equal(glue["step_ok"], ref["step_ok"])
    assert np.array_equal(glue["newton_its"], ref["newton_its"])
    assert np.array_equal(glue["sol_steps"], ref["sol_steps"])
    assert np.array_equal(glue["bc_mask"], ref["bc_mask"])


@pytest.mark.gpu
@needs_glue
@pytest.mark.parametrize("ci", [0, 1], ids=["flume101x11_100steps", "wetdry12_4steps"])
def test_gpu_newton_installed_in_the_reference_time_loop(ci):
    """fe_newton_gpu in adh_time_stepper[FE_NEWTON]: the reference's time_loop runs every
    step, each succeeds where the reference's succeeds, the state after the N steps is
    within 1e-8 relative (h, u, v) of the reference's, and every state on the way within
    1e-7 (two Newton solves stopped by the same tests still differ by what those tests
    allow: the reference accepts a step once the increment is below inc_nonlin)."""
    case = _cases()[ci]
    ref = run_harness("loop", case)
    gpu = run_harness("loop_gpu", case, binary=GLUE_HARNESS)
    assert np.array_equal(gpu["step_ok"], ref["step_ok"])
    n = 3 * case.nnodes
    a, b = gpu["sol_steps"].reshape(-1, n), ref["sol_steps"].reshape(-1, n)
    assert a.shape == b.shape == (case.nsteps, n)
    final = max(rel_err(a[-1], b[-1]))
    worst = max(max(rel_err(x, y)) for x, y in zip(a, b))
    assert final < 1e-8 and worst < 1e-7, (final, worst)
    assert np.array_equal(gpu["bc_mask"], ref["bc_mask"])
