"""The C-ABI library: it loads, exports every entry point include/*.h
declares, and fails loudly (error status, no fallback) when no GPU is
present.  CPU-only checks."""
import ctypes as C
import os
import re

import pytest

import openqcd_b200 as qb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    names = []
    inc = os.path.join(ROOT, "include")
    for f in sorted(os.listdir(inc)):
        if f.endswith(".h"):
            src = open(os.path.join(inc, f)).read()
            src = re.sub(r"/\*.*?\*/", " ", src, flags=re.S)
            for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\([^;{]*\)\s*;", src, re.M):
                if not m.group(0).lstrip().startswith("typedef"):
                    names.append(m.group(1))
    return names


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(qb.LIB_PATH):
        import importlib.util
        spec = importlib.util.spec_from_file_location("build", os.path.join(ROOT, "openqcd-2.4.2_b200", "build.py"))
        m = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(m)
        m.build()
    return qb.lib()


def test_header_declares_the_drop_in_names():
    names = set(declared())
    for n in ("Dw_dble", "Dwee_dble", "Dwoo_dble", "Dwoe_dble", "Dweo_dble", "Dwhat_dble", "Dw", "Dwee", "Dwoo",
              "Dwoe", "Dweo", "Dwhat", "apply_sw_dble", "apply_sw", "apply_swinv_dble", "sap", "sap_gcr"):
        assert n in names, n


def test_every_declared_symbol_is_exported(lib):
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_the_header():
    assert set(declared()) <= set(qb.EXPORTED) | {"b200_dev_free"}


def test_no_gpu_fails_loudly(lib):
    """Without a CUDA device the library reports an error; nothing computes
    on the CPU instead."""
    import shutil
    import subprocess
    import sys
    if shutil.which("nvidia-smi") and subprocess.run(["nvidia-smi"], capture_output=True).returncode == 0:
        pytest.skip("a GPU is present")
    code = ("import sys; sys.path.insert(0, %r); import openqcd_b200 as qb\n"
            "try:\n    qb.geometry((8,8,8,8),(4,4,4,4))\nexcept qb.B200Error as e:\n    print('ERR', e)\n"
            % os.path.join(ROOT, "openqcd-2.4.2_b200"))
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120)
    assert "ERR" in p.stdout, p.stdout + p.stderr
