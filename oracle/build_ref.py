"""Build recipe for the reference CPU oracle (test infrastructure only).

Compiles the reference's own C modules where they lie (read-only) together
with oracle/ref_driver.c into one shared library per lattice geometry:

    oracle/_ref/<tag>/libref.so      tag = "<L0>x<L1>x<L2>x<L3>_t<NTHREAD>"

The reference fixes its geometry at compile time in include/global.h
(NPROCx, Lx, Lx_TRD; include/global.h:18-36).  This recipe writes an edited
copy of that header into the (git-ignored) build folder -- NPROCx = 1 and the
requested sizes -- and force-includes it, so the original header is never
seen.  MPI is replaced by the serial stub in oracle/mpi_stub/mpi.h.

Flags follow the reference's devel Makefiles (devel/dirac/Makefile:88-90)
with c89 relaxed to gnu11 and -fPIC added.  One workaround: the reference
defines cm3x3_unityv() only in the non-x64 branch of
modules/su3fcts/cm3x3.c, so that file is compiled a second time without
-DAVX and only that one symbol is kept.

Usage:  python oracle/build_ref.py 8 8 8 8  4 4 4 8   [--ref PATH] [--portable]
"""
import argparse
import concurrent.futures as cf
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_REF = "/root/reference"
CFLAGS = ["-std=gnu11", "-O", "-fopenmp", "-fPIC", "-mfpmath=sse", "-mno-avx",
          "-DAVX", "-DFMA3", "-DPM", "-w"]


def tag_of(L, T, portable=False):
    vol = L[0] * L[1] * L[2] * L[3]
    nthr = vol // (T[0] * T[1] * T[2] * T[3])
    return "%dx%dx%dx%d_t%d%s" % (L[0], L[1], L[2], L[3], nthr, "_c" if portable else "")


def lib_path(L, T, portable=False):
    return os.path.join(HERE, "_ref", tag_of(L, T, portable), "libref.so")


def gen_global_h(ref, L, T, out):
    src = open(os.path.join(ref, "include", "global.h")).read()
    for i in range(4):
        src = re.sub(r"(#define NPROC%d )\d+" % i, r"\g<1>1", src)
        src = re.sub(r"(#define L%d )\d+" % i, r"\g<1>%d" % L[i], src)
        src = re.sub(r"(#define L%d_TRD )\d+" % i, r"\g<1>%d" % T[i], src)
    with open(out, "w") as f:
        # the MAIN_PROGRAM branch initialises pointers with NULL, and the
        # header is force-included ahead of any system header
        f.write("#include <stddef.h>\n" + src)


def run(cmd):
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError("failed: %s\n%s" % (" ".join(cmd), p.stderr[-4000:]))


def build(L, T, ref=DEFAULT_REF, jobs=None, verbose=True, portable=False):
    """portable=True compiles the reference's plain-C code paths (no -DAVX
    -DFMA3): identical algorithms, but the SAP minimal-residual step uses the
    exact reciprocal 1/r where the AVX path uses the approximate vrcpss
    instruction (modules/sap/blk_solv.c:291-300)."""
    out_dir = os.path.join(HERE, "_ref", tag_of(L, T, portable))
    lib = os.path.join(out_dir, "libref.so")
    gen = os.path.join(out_dir, "gen")
    obj = os.path.join(out_dir, "obj")
    os.makedirs(gen, exist_ok=True)
    os.makedirs(obj, exist_ok=True)
    gh = os.path.join(gen, "global.h")
    gen_global_h(ref, L, T, gh)
    inc = ["-include", gh, "-I", os.path.join(HERE, "mpi_stub"),
           "-I", os.path.join(ref, "include")]
    mods = []
    mdir = os.path.join(ref, "modules")
    for d in sorted(os.listdir(mdir)):
        if d == "nompi" or not os.path.isdir(os.path.join(mdir, d)):
            continue
        for f in sorted(os.listdir(os.path.join(mdir, d))):
            if f.endswith(".c"):
                mods.append(os.path.join(mdir, d, f))
    jobs = jobs or os.cpu_count() or 4
    cflags = [f for f in CFLAGS if f not in ("-DAVX", "-DFMA3", "-DPM")] if portable else CFLAGS
    cmds = []
    objs = []
    for m in mods:
        o = os.path.join(obj, os.path.basename(m)[:-2] + ".o")
        objs.append(o)
        if not (os.path.exists(o) and os.path.getmtime(o) > os.path.getmtime(gh)):
            cmds.append(["gcc"] + cflags + inc + ["-c", m, "-o", o])
    extra = []
    if not portable:
        # cm3x3_unityv workaround (see module docstring)
        cmx = os.path.join(obj, "cm3x3_noavx_full.o")
        cmk = os.path.join(obj, "cm3x3_unityv.o")
        flags_noavx = [f for f in CFLAGS if f not in ("-DAVX", "-DFMA3")]
        cmds.append(["gcc"] + flags_noavx + inc + ["-c", os.path.join(mdir, "su3fcts", "cm3x3.c"), "-o", cmx])
        extra = [cmk]
    drv = os.path.join(obj, "ref_driver.o")
    cmds.append(["gcc"] + cflags + ["-DMAIN_PROGRAM"] + inc +
                ["-c", os.path.join(HERE, "ref_driver.c"), "-o", drv])
    with cf.ThreadPoolExecutor(jobs) as ex:
        list(ex.map(run, cmds))
    if not portable:
        run(["objcopy", "--keep-global-symbol=cm3x3_unityv", cmx, cmk])
    run(["gcc", "-shared", "-fopenmp", "-Wl,-Bsymbolic", "-o", lib] + objs + extra + [drv, "-lm"])
    if verbose:
        print("built", lib)
    return lib


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("dims", type=int, nargs=8, help="L0 L1 L2 L3 L0_TRD L1_TRD L2_TRD L3_TRD")
    ap.add_argument("--ref", default=DEFAULT_REF)
    ap.add_argument("--portable", action="store_true")
    a = ap.parse_args()
    build(a.dims[:4], a.dims[4:], a.ref, portable=a.portable)


if __name__ == "__main__":
    sys.exit(main())
