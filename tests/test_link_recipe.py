"""The link recipe for openQCD programs, checked on the CPU: the reference
files that define one of the library's names are compiled with those names
renamed (-D<name>=ref_<name>), linked with every other reference module and
the library into one program, and in that program each of the library's
names that is called is resolved from the library (undefined in the
objects, never defined there) while the
functions the library does not replace (write_cnfg, dfl_update,
inv_pauli_dble, Dw_blk, ...) stay defined by the reference's objects."""
import os
import re
import shutil
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "openqcd-2.4.2_b200")
LIB = os.path.join(PKG, "libopenqcd_b200.so")
REF = "/root/reference"
sys.path.insert(0, os.path.join(ROOT, "oracle"))

# reference file -> the names the library provides (the integration table)
RENAMES = {
    "dirac/Dw.c": "Dw Dwee Dwoo Dwoe Dweo Dwhat",
    "dirac/Dw_dble.c": "Dw_dble Dwee_dble Dwoo_dble Dwoe_dble Dweo_dble Dwhat_dble",
    "sw_term/pauli.c": "apply_sw",
    "sw_term/pauli_dble.c": "apply_sw_dble apply_swinv_dble",
    "sap/sap.c": "sap",
    "sap/sap_gcr.c": "sap_gcr",
    "linsolv/fgcr.c": "fgcr",
    "linalg/salg.c": "spinor_prod spinor_prod_re norm_square mulc_spinor_add mulr_spinor_add scale normalize",
    "linalg/salg_dble.c": "spinor_prod_dble spinor_prod_re_dble norm_square_dble mulc_spinor_add_dble "
                          "mulr_spinor_add_dble scale_dble normalize_dble",
    "forces/tmcg.c": "tmcg tmcgeo",
    "forces/tmcgm.c": "tmcgm",
    "archive/archive.c": "export_cnfg import_cnfg",
    "archive/sarchive.c": "export_sfld import_sfld",
    "dfl/dfl_modes.c": "dfl_modes",
    "dfl/dfl_subspace.c": "dfl_s2vd dfl_vd2s dfl_subspace",
    "dfl/dfl_sap_gcr.c": "dfl_sap_gcr dfl_sap_gcr2",
    "dfl/ltl_gcr.c": "ltl_gcr",
    "little/Aw.c": "Aw Aweeinv Awooinv Awoe Aweo Awhat",
    "little/Aw_dble.c": "Aw_dble Aweeinv_dble Awooinv_dble Awoe_dble Aweo_dble Awhat_dble",
    "little/Aw_ops.c": "set_Aw set_Awhat",
    "little/ltl_modes.c": "set_ltl_modes ltl_matrix dfl_Lvd dfl_LRvd dfl_RLvd dfl_Lv",
}
KEPT = ["write_cnfg", "dfl_update", "inv_pauli_dble", "mul_pauli_dble", "Dw_blk", "blk_mres", "fgcr4vd"]

MAIN = r"""
#include <stdio.h>
#include "global.h"
#include "dirac.h"
#include "sap.h"
#include "dfl.h"
#include "archive.h"
#include "sw_term.h"
#include "linsolv.h"
#include "little.h"

int main(void)
{
   void *p[] = {(void *)Dw_dble, (void *)sap_gcr, (void *)dfl_sap_gcr, (void *)export_cnfg, (void *)apply_sw_dble,
                (void *)fgcr, (void *)Awhat_dble, (void *)set_Awhat, (void *)ltl_gcr, (void *)write_cnfg,
                (void *)dfl_update, (void *)inv_pauli_dble, (void *)Dw_blk, (void *)blk_mres, (void *)fgcr4vd};
   printf("%d\n", (int)(sizeof(p) / sizeof(p[0])));
   return 0;
}
"""


def test_library_names_come_from_the_library(tmp_path):
    if not (os.path.isdir(os.path.join(REF, "modules")) and os.path.exists(LIB) and shutil.which("gcc")):
        pytest.skip("reference sources, library or gcc missing")
    import build_ref
    L, T = (8, 8, 8, 8), (4, 4, 4, 8)
    objdir = os.path.join(os.path.dirname(build_ref.lib_path(list(L), list(T), True)), "obj")
    gh = os.path.join(os.path.dirname(objdir), "gen", "global.h")
    if not os.path.isdir(objdir) or not os.path.exists(gh):
        pytest.skip("portable reference objects not built")
    cflags = [f for f in build_ref.CFLAGS if f not in ("-DAVX", "-DFMA3", "-DPM")]
    inc = ["-include", gh, "-I", os.path.join(ROOT, "oracle", "mpi_stub"), "-I", os.path.join(REF, "include")]
    objs = []
    renamed = {os.path.basename(f)[:-2]: (f, names.split()) for f, names in RENAMES.items()}
    for o in sorted(os.listdir(objdir)):
        base = o[:-2]
        if not o.endswith(".o") or base == "ref_driver":
            continue
        if base in renamed:
            f, names = renamed[base]
            out = str(tmp_path / o)
            cmd = ["gcc"] + cflags + inc + ["-D%s=ref_%s" % (n, n) for n in names] + \
                  ["-c", os.path.join(REF, "modules", f), "-o", out]
            p = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
            assert p.returncode == 0, p.stderr[-2000:]
            objs.append(out)
        else:
            objs.append(os.path.join(objdir, o))
    src = tmp_path / "main.c"
    src.write_text(MAIN)
    mo = str(tmp_path / "main.o")
    p = subprocess.run(["gcc"] + cflags + ["-DMAIN_PROGRAM"] + inc + ["-c", str(src), "-o", mo],
                       capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr[-2000:]
    exe = str(tmp_path / "prog")
    p = subprocess.run(["gcc", "-fopenmp", "-o", exe, mo] + objs + ["-L", PKG, "-lopenqcd_b200", "-lm",
                                                                   "-Wl,-rpath," + PKG],
                       capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr[-3000:]
    nm = subprocess.run(["nm", exe], capture_output=True, text=True, timeout=60).stdout
    sym = {}
    for line in nm.splitlines():
        m = re.match(r"^\s*([0-9a-f]*)\s+(\w)\s+(\S+)$", line)
        if m:
            sym[m.group(3)] = m.group(2)
    used = 0
    for names in RENAMES.values():
        for n in names.split():
            # never defined by the objects: referenced from the library, or not referenced at all
            assert sym.get(n) in (None, "U"), (n, sym.get(n))
            used += sym.get(n) == "U"
            assert sym.get("ref_" + n) in ("T", "t"), n          # the reference's copy, renamed
    assert used >= 20        # the calls of the kept modules and of main resolve to the library
    for n in KEPT:
        assert sym.get(n) in ("T", "t"), n
