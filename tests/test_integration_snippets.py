"""The C snippets of INTEGRATION.md compile against the reference's own headers
(the structures they read: SMODEL_SUPER, SGRID, SLIN_SYS, the series API) and
include/adh_sw2_gpu.h, the way a maintainer would paste them into the reference."""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_SRC = "/root/reference/src"


def snippets():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    return re.findall(r"```c\n(.*?)```", text, flags=re.S)


@pytest.mark.skipif(not os.path.exists(os.path.join(REF_SRC, "include", "adh.h")) or shutil.which("gcc") is None,
                    reason="reference sources or gcc not present")
def test_integration_snippets_compile_against_the_reference(tmp_path):
    blocks = snippets()
    assert len(blocks) == 4
    init, set_step, newton, mass = blocks
    unit = ('#include "adh.h"\n' + init +
            "\nint gpu_step(SMODEL_SUPER *sm, int nsubsteps, int ivx, int ivy) {\n" + set_step + newton + "}\n"
            "\ndouble gpu_mass(SMODEL_SUPER *sm, double dt, double initial_grid_mass, double total_time_mass_flux) {\n"
            + mass + "    return grid_mass_error;\n}\n"
            "int use_all(SMODEL_SUPER *sm) { return sw2_gpu_init(sm) + gpu_step(sm, 1, 1, 2)"
            " + (gpu_mass(sm, 1.0, 0.0, 0.0) > 0); }\n")
    src = tmp_path / "glue.c"
    src.write_text(unit)
    incs = ["-I", os.path.join(ROOT, "oracle", "shim"), "-I", os.path.join(ROOT, "include")]
    for d, sub, _ in os.walk(REF_SRC):
        if "/test" not in d:
            incs += ["-I", d]
    incs += ["-I", os.path.join(REF_SRC, "test")]
    r = subprocess.run(["gcc", "-std=gnu99", "-fcommon", "-fsyntax-only", "-Werror=implicit-function-declaration",
                        "-Werror=incompatible-pointer-types", "-Werror=int-conversion", *incs, str(src)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "obj")) or shutil.which("gcc") is None,
                    reason="reference objects (oracle/_ref/obj) or gcc not present")
def test_reference_objects_and_library_link_together(tmp_path):
    """The glue, the reference's own objects and libadh_sw2_gpu.so link into one
    program with no clashing symbols (the library exports only sw2g_* / sw2n_*)."""
    from adh_kraken_b200 import capi
    if not os.path.exists(os.path.join(REF_SRC, "include", "adh.h")):
        pytest.skip("reference headers not present")
    init, set_step, newton, mass = snippets()
    glue = ('#include "adh.h"\nSADH_DEF adh_def;\n'
            "void sflags_init(SFLAGS *f) { memset(f, 0, sizeof(SFLAGS)); }\n" + init +
            "\nint gpu_step(SMODEL_SUPER *sm, int nsubsteps, int ivx, int ivy) {\n" + set_step + newton + "}\n"
            "int main(int argc, char **argv) { if (argc > 5) return sw2_gpu_init(NULL) + gpu_step(NULL, 1, 1, 2);"
            " return 0; }\n")
    src = tmp_path / "glue.c"
    src.write_text(glue)
    incs = ["-I", os.path.join(ROOT, "oracle", "shim"), "-I", os.path.join(ROOT, "include")]
    for d, sub, _ in os.walk(REF_SRC):
        if "/test" not in d:
            incs += ["-I", d]
    incs += ["-I", os.path.join(REF_SRC, "test")]
    objs = []
    for d, _, files in os.walk(os.path.join(ROOT, "oracle", "_ref", "obj")):
        objs += [os.path.join(d, f) for f in files if f.endswith(".o")]
    libdir = os.path.dirname(capi.LIB_PATH)
    exe = tmp_path / "glue"
    r = subprocess.run(["gcc", "-std=gnu99", "-fcommon", "-w", *incs, "-o", str(exe), str(src),
                        os.path.join(ROOT, "oracle", "shim", "ref_shim.c"), *objs, "-L", libdir, "-ladh_sw2_gpu",
                        "-Wl,-rpath," + libdir, "-lm"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert run.returncode == 0, run.stderr
