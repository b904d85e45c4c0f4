"""Build libopenqcd_b200.so in-tree for sm_100a with nvcc.

    python openqcd-2.4.2_b200/build.py [--verbose]

Every csrc/*.cu file is compiled separately (in parallel) with
-gencode arch=compute_100a,code=sm_100a -lineinfo -O3, then linked into one
shared library next to this file.  The CUDA runtime is linked statically so
the library has no dependency besides the driver.
"""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libopenqcd_b200.so")
NVCC = os.environ.get("NVCC", "nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
         "-Xcompiler", "-fPIC", "-Xcompiler", "-O2", "--expt-relaxed-constexpr",
         "-I", os.path.join(HERE, "..", "include")]


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))


def headers_mtime():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(HERE, "..", "include", "openqcd_b200.h"))
    return max(os.path.getmtime(h) for h in hs)


def compile_one(src, extra, verbose):
    o = os.path.join(OBJ, src[:-3] + ".o")
    s = os.path.join(CSRC, src)
    if os.path.exists(o) and os.path.getmtime(o) > max(os.path.getmtime(s), headers_mtime()):
        return o
    cmd = [NVCC] + FLAGS + extra + ["-c", s, "-o", o]
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError("nvcc failed on %s:\n%s" % (src, p.stdout + p.stderr))
    if verbose and (p.stdout or p.stderr):
        print(p.stdout + p.stderr)
    return o


def build(verbose=False, extra=None):
    os.makedirs(OBJ, exist_ok=True)
    extra = list(extra or [])
    if verbose:
        extra += ["-Xptxas", "-v"]
    with cf.ThreadPoolExecutor(min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: compile_one(s, extra, verbose), sources()))
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-Xlinker", "-Bsymbolic",
               "-o", LIB] + objs
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode != 0:
            raise RuntimeError("link failed:\n" + p.stdout + p.stderr)
    return LIB


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv))
