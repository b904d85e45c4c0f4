"""The allocation-free Dwhat_dble entry point (b200_dev_Dwhat_dble_noalloc).

It exists for callers that cannot let the library allocate device memory (CUDA
graph capture, a device memory pool that owns all memory, loops that must not
synchronise on cudaMalloc).  Its odd-site intermediate lives in a static device
array instead of a cudaMalloc'd buffer, so its output must equal the regular
Dwhat_dble entry point's (same kernels, same arithmetic) call after call, and
lattices larger than the array must be refused.

This file is collected last so that a run stopping at the first failure has
run every other test before it; it needs nothing from them.
"""
import numpy as np
import pytest

import openqcd_b200 as qb
from helpers import Setup, site_rel_err

pytestmark = pytest.mark.gpu


def test_noalloc_matches_dwhat_twice():
    st = Setup((8, 8, 8, 8), (4, 4, 4, 4), eps=0.4, csw=1.5, m0=-0.05)
    L = qb.lib()
    mu = 0.137
    s = qb.DevField(64).from_ref(st.source(77))
    r_ref = qb.DevField(64)
    qb.dev_dirac("Dwhat", mu, s, r_ref)
    want = r_ref.to_ref(st.vol)
    for _ in range(2):   # two calls in a row reuse the shared static array
        r = qb.DevField(64)
        qb.check(L.b200_dev_Dwhat_dble_noalloc(mu, s.ptr, r.ptr))
        got = r.to_ref(st.vol)
        assert site_rel_err(got, want, st.vol) <= 1e-13
        r.free()


def test_noalloc_rejects_large_lattice():
    L = qb.lib()
    qb.geometry((32, 32, 16, 16), (4, 4, 4, 4))      # 262144 sites > 131072
    qb.set_parms(1.5, 0.0)
    qb.random_ud(0.3, 5)
    qb.sw_term()
    s = qb.DevField(64).random(1.0, 1)
    r = qb.DevField(64)
    rc = L.b200_dev_Dwhat_dble_noalloc(0.0, s.ptr, r.ptr)
    assert rc == -1
    assert "131072" in L.b200_last_error().decode()
