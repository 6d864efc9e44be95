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


def test_headers_compile_as_c99_and_cxx(tmp_path):
    """The reference is C99: both headers must compile in a C99 and a C++ unit as the
    reference-side caller would include them."""
    import shutil
    import subprocess
    import pytest
    src = tmp_path / "use.c"
    src.write_text('#include "adh_sw2_gpu.h"\n#include "adh_sw2_gnn.h"\n'
                   "int use(sw2g_model *m) { double out[2]; return sw2g_grid_mass(m, 0, 1.0, 1.0, out, 0); }\n")
    inc = os.path.join(ROOT, "include")
    for cc, std in (("gcc", "-std=c99"), ("g++", "-std=c++17")):
        if shutil.which(cc) is None:
            pytest.skip(f"{cc} not available")
        lang = ["-x", "c++"] if cc == "g++" else []
        r = subprocess.run([cc, std, "-Wall", "-Wextra", "-Werror", "-pedantic", "-fsyntax-only", "-I", inc,
                            *lang, str(src)], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr


def test_no_cpu_fallback_without_a_gpu():
    """Without a usable GPU the model constructor fails with the CUDA error; nothing
    falls back to a CPU path."""
    import pytest
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from adh_kraken_b200.capi import SW2Error, SW2Model
    from adh_kraken_b200.mesh import small_delaunay_case
    with pytest.raises(SW2Error, match="cuda|CUDA"):
        SW2Model(small_delaunay_case(n=12, seed=5))
