"""The allocation-free Dwhat_dble entry point (b200_dev_Dwhat_dble_noalloc).

It exists for callers that cannot let the library allocate device memory: an
application whose own memory pool already holds the device, or a service
whose device footprint must stay fixed after start-up.  Its odd-site
intermediate lives in a static device array instead of a cudaMalloc'd
buffer, so its output must equal the regular Dwhat_dble entry point's (same
kernels, same arithmetic) call after call, the device's free memory must
not change across its calls, and lattices larger than the array must be
refused.

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


def test_noalloc_allocates_nothing():
    """In a fresh geometry (the regular Dwhat's scratch not yet allocated)
    the device's free memory is the same before and after two calls; the
    result then equals the regular entry point's."""
    torch = pytest.importorskip("torch")
    L = qb.lib()
    # first call on this device in a throwaway geometry: it loads the
    # array's module and looks up its address, which is set-up, not a
    # per-call allocation
    qb.geometry((8, 8, 8, 8), (4, 4, 4, 4), qb.even_first_ipt((8, 8, 8, 8)))
    qb.set_parms(1.5, -0.05)
    qb.random_ud(0.4, 3)
    qb.sw_term()
    a = qb.DevField(64).random(1.0, 2)
    b = qb.DevField(64)
    qb.check(L.b200_dev_Dwhat_dble_noalloc(0.1, a.ptr, b.ptr))
    a.free(); b.free()

    qb.geometry((8, 8, 8, 16), (4, 4, 4, 4), qb.even_first_ipt((8, 8, 8, 16)))
    qb.set_parms(1.7, -0.05)
    qb.random_ud(0.3, 4)
    qb.sw_term()
    vol = L.b200_volume()
    s = qb.DevField(64).random(1.0, 5)
    r = qb.DevField(64)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(2):
        qb.check(L.b200_dev_Dwhat_dble_noalloc(0.137, s.ptr, r.ptr))
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert free1 == free0, "free device memory changed by %d bytes" % (free0 - free1)
    got = r.to_ref(vol)
    want = qb.DevField(64)
    qb.dev_dirac("Dwhat", 0.137, s, want)
    assert site_rel_err(got, want.to_ref(vol), vol) <= 1e-13


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
