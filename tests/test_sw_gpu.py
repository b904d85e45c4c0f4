"""Parity of the device SW term (construction, inversion, site-local
application) with the reference (modules/sw_term/sw_term.c, pauli_dble.c,
pauli.c)."""
import numpy as np
import pytest

import openqcd_b200 as qb
from helpers import Setup, site_rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    return Setup((8, 8, 8, 8), (4, 4, 4, 4), eps=0.4, csw=1.5, m0=-0.05)


def pauli_rel_err(a, b):
    a = np.asarray(a).reshape(-1, 36)
    b = np.asarray(b).reshape(-1, 36)
    return float((np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)).max())


def test_sw_term_from_links(setup):
    """sw_term(NO_PTS) on the device from the uploaded links equals the
    reference's SW field (clover field tensor + pauli_term + 4+m0)."""
    qb.upload_ud(setup.ud)
    assert qb.sw_term() == 0
    dev = qb.download_swd(setup.vol, 0)
    assert pauli_rel_err(dev, setup.swd) <= 1e-14
    qb.upload_swd(setup.swd)


def test_sw_inverse(setup):
    """The device inverse equals the reference's sw_term(ALL_PTS)."""
    setup.ref.sw_term(3)
    ref_inv = setup.ref.swd()
    setup.ref.sw_term(0)
    dev_inv = qb.download_swd(setup.vol, 1)
    assert pauli_rel_err(dev_inv, ref_inv) <= 1e-12


@pytest.mark.parametrize("mu", [0.0, 0.31])
def test_apply_sw_dble(setup, mu):
    s = setup.source(5)
    r_ref = setup.ref.apply_sw_dble(setup.vol, mu, setup.swd, s)
    r_dev = qb.apply_sw_dble(setup.vol, mu, setup.swd, s)
    assert site_rel_err(r_dev, r_ref, setup.vol) <= 1e-14


def test_apply_sw_single(setup):
    s = setup.source(6).astype(np.float32)
    m = setup.swd.astype(np.float32)
    r_ref = setup.ref.apply_sw(setup.vol, 0.2, m, s)
    r_dev = qb.apply_sw(setup.vol, 0.2, m, s)
    assert site_rel_err(r_dev, r_ref, setup.vol) <= 2e-6


@pytest.mark.parametrize("mu", [0.0, 0.25])
def test_apply_swinv_dble(setup, mu):
    s = setup.source(7)
    r_ref, f_ref = setup.ref.apply_swinv_dble(setup.vol, mu, setup.swd, s)
    r_dev, f_dev = qb.apply_swinv_dble(setup.vol, mu, setup.swd, s)
    assert f_ref == 0 and f_dev == 0
    assert site_rel_err(r_dev, r_ref, setup.vol) <= 1e-12


def _pauli(diag, off=0.0):
    u = np.zeros(36)
    u[:6] = diag
    u[6:] = off
    return u


@pytest.mark.parametrize("diag,unsafe", [([1, 1, 1, 1, 1, 0.1], 0), ([1, 1, 1, 1, 1, 1e-3], 1),
                                          ([2, 1.5, 1, 1, 3, 0.5], 0)])
def test_inversion_safety_flag(setup, diag, unsafe):
    """The Frobenius-condition safety flag (pauli_dble.c:55-59) agrees with the
    reference on well and badly conditioned matrices."""
    m = np.concatenate([_pauli(diag, 0.01), _pauli(diag[::-1], 0.0)])
    s = np.ones(24)
    _, f_ref = setup.ref.apply_swinv_dble(1, 0.0, m, s)
    _, f_dev = qb.apply_swinv_dble(1, 0.0, m, s)
    assert f_ref == unsafe
    assert f_dev == unsafe
