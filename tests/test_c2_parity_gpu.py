"""Parity of the device operators with the reference on the single-operator
bandwidth configuration: a 32^3x64 lattice, links exp(0.3 X) from the
reference's own random_alg + expXsu3 (modules/linalg/liealg.c:289,
modules/su3fcts/chexp.c:878), m0 = -0.05, csw = 1.7, periodic gauge field
with antiperiodic quark time boundary (bc type 3), 4^4 blocks.

The reference's Dw_dble, Dwhat_dble (modules/dirac/Dw_dble.c:1377, :1792),
Dw and Dwhat (modules/dirac/Dw.c:973, :1378), run on the CPU from
oracle/_ref/64x32x32x32_*, are applied to the reference's field and
Gaussian source; the library gets the same field and SW term through its
drop-in entry points.  Bars, per-site relative spinor difference: 1e-13 for
FP64 and 2e-6 for FP32.  This is the lattice and field of the bench's
headline number.
"""
import numpy as np
import pytest

import openqcd_b200 as qb
import reflib
from helpers import Setup, site_rel_err

pytestmark = pytest.mark.gpu

TOL64 = 1e-13
TOL32 = 2e-6
L = (64, 32, 32, 32)


@pytest.fixture(scope="module")
def c2():
    if not reflib.ensure_built(L):
        pytest.skip("reference oracle for 32^3x64 is not built")
    st = Setup(L, (4, 4, 4, 4), eps=0.3, csw=1.7, m0=-0.05, seed=20251203)
    assert st.sw_fail == 0
    return st


@pytest.mark.parametrize("mu", [0.0, 0.137])
def test_c2_dw_dble(c2, mu):
    s = c2.source(101)
    r_ref = c2.ref.dirac_dble(0, mu, s)
    r_dev = qb.dirac_ref("Dw", 64, mu, s)
    err = site_rel_err(r_dev, r_ref, c2.vol)
    assert err <= TOL64, "Dw_dble mu=%g on 32^3x64: per-site rel err %.3e" % (mu, err)


def test_c2_dw_dble_unstaged(c2):
    """the direct-read FP64 kernel (SW matrices not staged) on the same case"""
    s = c2.source(102)
    r_ref = c2.ref.dirac_dble(0, 0.0, s)
    prev = qb.set_dw_staged(0)
    try:
        r_dev = qb.dirac_ref("Dw", 64, 0.0, s)
    finally:
        qb.set_dw_staged(prev)
    assert site_rel_err(r_dev, r_ref, c2.vol) <= TOL64


def test_c2_dwhat_dble(c2):
    s = c2.source(103)
    r0 = c2.source(104)
    c2.ref.sw_term(2)              # the reference's Dwhat needs the odd SW term inverted
    try:
        r_ref = c2.ref.dirac_dble(5, 0.0, s, r0)
    finally:
        c2.ref.sw_term(0)
    r_dev = qb.dirac_ref("Dwhat", 64, 0.0, s, r0)
    err = site_rel_err(r_dev, r_ref, c2.vol)
    assert err <= TOL64, "Dwhat_dble on 32^3x64: per-site rel err %.3e" % err


def test_c2_dw_single(c2):
    s = c2.source(105).astype(np.float32)
    r_ref = c2.ref.dirac(0, 0.0, s)
    r_dev = qb.dirac_ref("Dw", 32, 0.0, s)
    err = site_rel_err(r_dev, r_ref, c2.vol)
    assert err <= TOL32, "Dw on 32^3x64: per-site rel err %.3e" % err


def test_c2_dwhat_single(c2):
    s = c2.source(106).astype(np.float32)
    r0 = c2.source(107).astype(np.float32)
    c2.ref.sw_term(2)
    try:
        r_ref = c2.ref.dirac(5, 0.0, s, r0)
    finally:
        c2.ref.sw_term(0)
    r_dev = qb.dirac_ref("Dwhat", 32, 0.0, s, r0)
    err = site_rel_err(r_dev, r_ref, c2.vol)
    assert err <= TOL32, "Dwhat on 32^3x64: per-site rel err %.3e" % err


def test_c2_device_sw_term(c2):
    """the SW term built on the device from the uploaded links equals the
    reference's sw_term (the bench builds it this way)"""
    qb.sw_term()
    try:
        sw_dev = qb.download_swd(c2.vol)
        d = np.abs(sw_dev - c2.swd).max()
        assert d <= 1e-13 * np.abs(c2.swd).max(), d
        s = c2.source(108)
        r_ref = c2.ref.dirac_dble(0, 0.0, s)
        r_dev = qb.dirac_ref("Dw", 64, 0.0, s)
        assert site_rel_err(r_dev, r_ref, c2.vol) <= TOL64
    finally:
        qb.upload_swd(c2.swd)


def test_c2_block_orders(c2):
    """every block traversal order gives the same, bit-identical result (the
    order only changes when a block's face data are read)"""
    s = c2.source(109)
    r_ref = c2.ref.dirac_dble(0, 0.0, s)
    prev = qb.set_block_order(0)
    try:
        out = []
        for kind in range(5):
            qb.set_block_order(kind)
            out.append(qb.dirac_ref("Dw", 64, 0.0, s))
        k, ms = qb.tune_block_order()
        assert 0 <= k < 5 and all(t > 0 for t in ms)
    finally:
        qb.set_block_order(prev)
    assert site_rel_err(out[0], r_ref, c2.vol) <= TOL64
    for o in out[1:]:
        assert np.array_equal(o, out[0])
