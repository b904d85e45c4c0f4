"""Parity of the device Wilson-Dirac operators with the reference.

The reference's own Dw_dble/Dw and even-odd pieces (modules/dirac/Dw_dble.c,
Dw.c), run on the CPU from oracle/_ref, are applied to the same gauge field,
SW term and Gaussian source as the library's drop-in entry points.  Bars
(per-site relative spinor difference): 1e-13 for FP64, 2e-6 for FP32.
"""
import numpy as np
import pytest

import openqcd_b200 as qb
from helpers import OPS, Setup, site_rel_err

pytestmark = pytest.mark.gpu

TOL64 = 1e-13
TOL32 = 2e-6


@pytest.fixture(scope="module", params=[((8, 8, 8, 8), (4, 4, 4, 4)), ((16, 8, 8, 8), (4, 4, 4, 4))],
                ids=["8x8x8x8", "16x8x8x8"])
def setup(request):
    L, bs = request.param
    return Setup(L, bs, eps=0.4, csw=1.5 if L == (8, 8, 8, 8) else 1.7, m0=-0.05)


@pytest.mark.parametrize("op", OPS)
@pytest.mark.parametrize("mu", [0.0, 0.137])
def test_dirac_dble(setup, op, mu):
    s = setup.source(11)
    r0 = setup.source(12)          # the eo pieces keep or update one parity of r
    k = OPS.index(op)
    if op == "Dwhat":
        setup.ref.sw_term(2)       # reference needs the odd SW term inverted
    r_ref = setup.ref.dirac_dble(k, mu, s, r0)
    if op == "Dwhat":
        setup.ref.sw_term(0)
    r_dev = qb.dirac_ref(op, 64, mu, s, r0)
    err = site_rel_err(r_dev, r_ref, setup.vol)
    assert err <= TOL64, "%s_dble mu=%g: per-site rel err %.3e" % (op, mu, err)


@pytest.mark.parametrize("op", OPS)
def test_staged_equals_direct(setup, op):
    """The FP64 operators with bulk-staged SW matrices (the default) against
    the direct-read kernel: the same arithmetic."""
    s = setup.source(13)
    r0 = setup.source(14)
    prev = qb.set_dw_staged(0)
    try:
        out = []
        for mode in (0, 1):
            qb.set_dw_staged(mode)
            out.append(qb.dirac_ref(op, 64, 0.137, s, r0))
    finally:
        qb.set_dw_staged(prev)
    assert site_rel_err(out[1], out[0], setup.vol) <= 1e-15


@pytest.mark.parametrize("op", OPS)
def test_dirac_single(setup, op):
    mu = 0.137
    s = setup.source(21).astype(np.float32)
    r0 = setup.source(22).astype(np.float32)
    k = OPS.index(op)
    if op == "Dwhat":
        setup.ref.sw_term(2)
    r_ref = setup.ref.dirac(k, mu, s, r0)
    if op == "Dwhat":
        setup.ref.sw_term(0)
    r_dev = qb.dirac_ref(op, 32, mu, s, r0)
    err = site_rel_err(r_dev, r_ref, setup.vol)
    assert err <= TOL32, "%s mu=%g: per-site rel err %.3e" % (op, mu, err)


def test_twisted_mass_eo_flag(setup):
    """With the twisted-mass eo flag the odd-site mu is switched off
    (Dw_dble.c:1392-1395)."""
    mu = 0.2
    s = setup.source(31)
    setup.ref.set_tm_parms(1)
    qb.lib().b200_set_tm_parms(1)
    try:
        r_ref = setup.ref.dirac_dble(0, mu, s)
        r_dev = qb.dirac_ref("Dw", 64, mu, s)
        r_ref_oo = setup.ref.dirac_dble(2, mu, s)
        r_dev_oo = qb.dirac_ref("Dwoo", 64, mu, s)
    finally:
        setup.ref.set_tm_parms(0)
        qb.lib().b200_set_tm_parms(0)
    assert site_rel_err(r_dev, r_ref, setup.vol) <= TOL64
    assert site_rel_err(r_dev_oo, r_ref_oo, setup.vol) <= TOL64


def test_eo_decomposition(setup):
    """Dw = Dwee + Dwoo + Dwoe + Dweo on the device (devel/dirac/check6)."""
    mu = 0.05
    s = setup.source(41)
    full = qb.dirac_ref("Dw", 64, mu, s)
    z = np.zeros_like(s)
    even = qb.dirac_ref("Dwee", 64, mu, s, z)
    even = qb.dirac_ref("Dweo", 64, mu, -s, even)   # Dweo subtracts D_eo s from r
    odd = qb.dirac_ref("Dwoo", 64, mu, s, z) + qb.dirac_ref("Dwoe", 64, mu, s, z)  # both assign r_o
    vh = setup.vol // 2 * 24
    r = np.concatenate([even[:vh], odd[vh:]])
    assert site_rel_err(r, full, setup.vol) <= 1e-13


def test_gamma5_hermiticity(setup):
    """(g5 Dw(mu))^dag = g5 Dw(-mu): (g5 Dw(mu) s, t) = (s, g5 Dw(-mu) t)."""
    mu = 0.1
    s = setup.source(51)
    t = setup.source(52)
    vol = setup.vol

    def g5(x):
        y = x.reshape(vol, 4, 6).copy()
        y[:, 2:, :] *= -1
        return y.reshape(-1)

    def cdot(a, b):
        a = a.reshape(-1, 2)
        b = b.reshape(-1, 2)
        return complex(np.sum(a[:, 0] * b[:, 0] + a[:, 1] * b[:, 1]), np.sum(a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]))

    lhs = cdot(g5(qb.dirac_ref("Dw", 64, mu, s)), t)
    rhs = cdot(s, g5(qb.dirac_ref("Dw", 64, -mu, t)))
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_device_layout_roundtrip(setup):
    s = setup.source(61)
    f = qb.DevField(64).from_ref(s)
    back = f.to_ref(setup.vol)
    assert np.array_equal(back, s)
    g = qb.DevField(32).from_ref(s.astype(np.float32))
    assert np.array_equal(g.to_ref(setup.vol), s.astype(np.float32))


def test_gauge_roundtrip(setup):
    back = qb.download_ud(setup.vol)
    assert np.array_equal(back, setup.ud)
