"""The C-ABI library loads and exports every entry point include/adh_sw2_gpu.h
declares (no GPU needed to dlopen it)."""
import ctypes
import os
import re

from adh_kraken_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names |= set(re.findall(r"\b(sw2[gn]_[a-z0-9_]+)\s*\(", src))
    return names


def test_header_and_binding_agree():
    assert declared_symbols() == set(capi.EXPORTED)


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(capi.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_default_options_match_reference_defaults():
    o = capi.default_opts()
    # smodel_super_alloc_init.c: tol_nonlin 1e-8, inc_nonlin 1e-6, 10 iterations, 5 line-search cuts;
    # bcgstab_solver.c:20-21 tolerance 1e-11
    assert (o.tol_nonlin, o.inc_nonlin, o.max_nonlin_it, o.max_linesearch_cuts) == (1e-8, 1e-6, 10, 5)
    assert o.krylov_tol == 1e-11 and o.krylov_precision == 64 and o.use_guess == 0
