"""Dw_dble and Dw on page-locked host arrays run as a pipeline (copy in,
operator and copy out of different parts of the lattice overlap) when the
storage order has contiguous x0-pieces in each parity half, as openQCD's
ipt[] has for pieces of L0_TRD planes (here the reference build's own ipt
with L0_TRD = 4) and a lexicographic order for single planes.  Results:
equal to the whole-field path bit for bit, and to the reference's operator
to 1e-13 (FP64) / 2e-6 (FP32), also in place."""
import numpy as np
import pytest

import openqcd_b200 as qb
from helpers import Setup, site_rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    return Setup((16, 8, 8, 8), (4, 4, 4, 4), eps=0.4, csw=1.7, m0=-0.05)


def test_slab_plan(setup):
    assert qb.pipeline_slabs() == 4                # block rows of 16x8x8x8 with 4^4 blocks
    assert qb.pipeline_pieces() >= 3


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


def _piped_whole_inplace(prec, mu, s):
    dt = np.float64 if prec == 64 else np.float32
    f = qb.lib().Dw_dble if prec == 64 else qb.lib().Dw
    n = s.size
    hs, hr, hx = qb.HostArray(n, dt), qb.HostArray(n, dt), qb.HostArray(n, dt)
    try:
        hs.a[:] = s
        f(mu, hs.ptr, hr.ptr)
        assert qb.pipeline_used() == 1
        piped = hr.a.copy()
        prev = qb.set_pipeline(False)
        try:
            hr.a[:] = 0
            f(mu, hs.ptr, hr.ptr)
            assert qb.pipeline_used() == 0
            whole = hr.a.copy()
        finally:
            qb.set_pipeline(prev)
        hx.a[:] = s
        f(mu, hx.ptr, hx.ptr)
        assert qb.pipeline_used() == 1
        inplace = hx.a.copy()
    finally:
        for h in (hs, hr, hx):
            h.free()
    return piped, whole, inplace


@pytest.mark.parametrize("bs0", [4, 2])
@pytest.mark.parametrize("prec", [64, 32])
def test_pipelined_dw_plane_pieces(bs0, prec):
    """a lexicographic even-first storage order: pieces of one plane, four
    (bs0 = 4) or two (bs0 = 2) per block row; device-made fields"""
    L = (16, 8, 8, 8)
    qb.geometry(L, (bs0, 4, 4, 4), qb.even_first_ipt(L))
    qb.set_parms(1.7, -0.05, 0)
    qb.set_bc_theta((0.0, 0.0, 0.0))
    qb.random_ud(0.4, 11)
    assert qb.sw_term() == 0
    assert qb.pipeline_pieces() == 16 and qb.pipeline_slabs() == 16 // bs0
    dt = np.float64 if prec == 64 else np.float32
    s = np.random.default_rng(5).standard_normal(16 * 8 * 8 * 8 * 24).astype(dt)
    piped, whole, inplace = _piped_whole_inplace(prec, 0.07, s)
    assert np.abs(whole).max() > 0
    assert np.array_equal(piped, whole)
    assert np.array_equal(inplace, piped)


def test_pipelined_dw_pieces_thicker_than_rows(setup):
    """the reference build's ipt (pieces of L0_TRD = 4 planes) with blocks
    two planes thick: every piece spans two block rows"""
    L = (16, 8, 8, 8)
    qb.geometry(L, (2, 4, 4, 4), setup.ipt)
    qb.set_parms(1.7, -0.05, 0)
    qb.random_ud(0.4, 12)
    assert qb.sw_term() == 0
    assert qb.pipeline_slabs() == 8
    npc = qb.pipeline_pieces()
    assert 3 <= npc < 8
    s = np.random.default_rng(6).standard_normal(16 * 8 * 8 * 8 * 24)
    piped, whole, inplace = _piped_whole_inplace(64, 0.03, s)
    assert np.array_equal(piped, whole)
    assert np.array_equal(inplace, piped)
