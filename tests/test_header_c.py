"""The C boundary as an openQCD program sees it (no GPU needed).

1. include/openqcd_b200.h compiles after the reference's own headers
   (su3.h, dirac.h, sw_term.h, sap.h, linsolv.h, dfl.h, little.h, archive.h,
   linalg.h, sflds.h, forces.h, uflds.h): every drop-in name is declared
   twice, and C rejects a second declaration whose prototype differs
   ("conflicting types"), so the prototypes are the reference's.
2. A C program that includes only the header links against the library and
   runs: with b200_set_fatal(0) a call that needs a GPU returns an error
   code and a message instead of falling back to the CPU."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")
PKG = os.path.join(ROOT, "openqcd-2.4.2_b200")
LIB = os.path.join(PKG, "libopenqcd_b200.so")
REF_INC = "/root/reference/include"

pytestmark = pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc missing")

REF_HEADERS = ["su3.h", "dirac.h", "sw_term.h", "sap.h", "linsolv.h", "dfl.h", "little.h", "archive.h",
               "linalg.h", "sflds.h", "forces.h", "uflds.h"]


def test_header_matches_reference_prototypes(tmp_path):
    if not os.path.isdir(REF_INC):
        pytest.skip("reference headers not present")
    src = tmp_path / "both.c"
    src.write_text("".join('#include "%s"\n' % h for h in REF_HEADERS) +
                   '#include "openqcd_b200.h"\nint main(void) { return 0; }\n')
    p = subprocess.run(["gcc", "-std=gnu11", "-fopenmp", "-c", str(src), "-o", str(tmp_path / "both.o"),
                        "-I", INC, "-I", REF_INC, "-I", os.path.join(ROOT, "oracle", "mpi_stub")],
                       capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr[-3000:]
    assert "conflicting types" not in p.stderr


PROG = r"""
#include <stdio.h>
#include "openqcd_b200.h"

int main(void)
{
   void (*dw)(double, spinor_dble *, spinor_dble *) = Dw_dble;
   double (*sg)(int, int, int, double, double, spinor_dble *, spinor_dble *, int *, int *) = sap_gcr;
   int rc;

   b200_set_fatal(0);
   rc = b200_set_device(0);
   printf("set_device %d %s\n", rc, rc ? b200_last_error() : "ok");
   return (dw != 0 && sg != 0) ? 0 : 1;
}
"""


def test_c_program_links_and_runs(tmp_path):
    if not os.path.exists(LIB):
        pytest.skip("library not built")
    src = tmp_path / "prog.c"
    src.write_text(PROG)
    exe = tmp_path / "prog"
    p = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", str(src), "-o", str(exe), "-I", INC, "-L", PKG,
                        "-lopenqcd_b200", "-Wl,-rpath," + PKG], capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr[-3000:]
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("set_device ")
