"""Dw_dble and Dw on page-locked host arrays run as a pipeline over x0-slabs
(copy in, operator and copy out of different slabs overlap) when the
storage order has contiguous x0-slabs in each parity half, as openQCD's
ipt[] has for slabs of L0_TRD planes (here the reference build's own ipt
with L0_TRD = 4).  Results: equal to the whole-field path bit for bit, and
to the reference's operator to 1e-13 (FP64) / 2e-6 (FP32), also in place."""
import numpy as np
import pytest

import openqcd_b200 as qb
from helpers import Setup, site_rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    return Setup((16, 8, 8, 8), (4, 4, 4, 4), eps=0.4, csw=1.7, m0=-0.05)


def test_slab_plan(setup):
    assert qb.pipeline_slabs() >= 3


@pytest.mark.parametrize("prec", [64, 32])
def test_pipelined_dw(setup, prec):
    dt = np.float64 if prec == 64 else np.float32
    f = qb.lib().Dw_dble if prec == 64 else qb.lib().Dw
    mu = 0.07
    s = setup.source(61).astype(dt)
    n = setup.vol * 24
    hs, hr, hx = qb.HostArray(n, dt), qb.HostArray(n, dt), qb.HostArray(n, dt)
    try:
        hs.a[:] = s
        f(mu, hs.ptr, hr.ptr)
        piped = hr.a.copy()
        prev = qb.set_pipeline(False)
        try:
            hr.a[:] = 0
            f(mu, hs.ptr, hr.ptr)
            whole = hr.a.copy()
        finally:
            qb.set_pipeline(prev)
        assert np.array_equal(piped, whole)
        hx.a[:] = s
        f(mu, hx.ptr, hx.ptr)                        # in place
        assert np.array_equal(hx.a, piped)
    finally:
        for h in (hs, hr, hx):
            h.free()
    if prec == 64:
        ref = setup.ref.dirac_dble(0, mu, s)
        assert site_rel_err(piped, ref, setup.vol) <= 1e-13
    else:
        ref = setup.ref.dirac(0, mu, s)
        assert site_rel_err(piped, ref, setup.vol) <= 2e-6
