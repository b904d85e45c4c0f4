"""Failure paths of the device code, made without a GPU fault.

- The bounded waits of the bulk-copy kernels: a self-check kernel waits, with
  a short poll limit, on an mbarrier that nothing completes; the wait gives
  up, the host reads the error status, and the context stays usable.
- sap_gcr's ifail = -3 (modules/sap/sap_gcr.c:60-78, :205): an SW field with
  one odd-site Pauli block whose inversion is not safe (Frobenius condition
  above the reference's bound, pauli_dble.c) is uploaded from the host;
  sap_gcr with the even-odd block solver then returns ifail = -3, psi = 0
  and the norm of the source, as the reference documents.
"""
import numpy as np
import pytest

import openqcd_b200 as qb
from helpers import Setup, site_rel_err

pytestmark = pytest.mark.gpu

BS = (4, 4, 4, 4)


@pytest.fixture(scope="module")
def setup():
    return Setup((8, 8, 8, 8), BS, eps=0.4, csw=1.5, m0=0.0)


def test_bounded_wait_gives_up_and_context_survives(setup):
    L = qb.lib()
    rc = L.b200_selfcheck_bounded_wait(2000)
    assert rc == -1
    assert "gave up waiting" in L.b200_last_error().decode()
    assert L.b200_sync() == 0            # the flag was read and cleared
    # the context still runs kernels and gives the reference's result
    s = setup.source(3)
    r_dev = qb.dirac_ref("Dw", 64, 0.1, s)
    r_ref = setup.ref.dirac_dble(0, 0.1, s)
    assert site_rel_err(r_dev, r_ref, setup.vol) <= 1e-13


def test_bounded_wait_limit_checked(setup):
    L = qb.lib()
    assert L.b200_selfcheck_bounded_wait(0) == -1
    assert "limit" in L.b200_last_error().decode()
    assert L.b200_selfcheck_bounded_wait(1 << 23) == -1


def _unsafe(swd, vol, site):
    """copy of the SW field with the upper Pauli block of storage site
    `site` replaced by a badly conditioned one (diagonal 1, 1, 1, 1, 1, 1e-3)"""
    m = swd.reshape(2 * vol, 36).copy()
    u = np.zeros(36)
    u[:6] = [1, 1, 1, 1, 1, 1e-3]
    u[6:] = 0.01
    m[2 * site] = u
    return m.reshape(-1)


@pytest.mark.parametrize("istop", [0, 1])
def test_sap_gcr_unsafe_odd_sw_term(setup, istop):
    vol = setup.vol
    eta = setup.source(5)
    qb.set_sap_parms(BS, 1, 4, 5)
    try:
        flag = qb.upload_swd(_unsafe(setup.swd, vol, vol // 2 + 17))    # an odd site
        assert flag & 2
        psi, rho, ifail, st = qb.sap_gcr(16, 256, istop, 1e-10, 0.0, eta)
        assert ifail == -3 and st == 0
        assert not psi.any()
        e = eta.reshape(vol, 24)
        want = np.sqrt((e ** 2).sum(axis=1)).max() if istop else np.linalg.norm(eta)
        assert abs(rho - want) <= 1e-12 * want
    finally:
        assert qb.upload_swd(setup.swd) == 0
    # with the SW field restored the solver runs again
    psi, rho, ifail, st = qb.sap_gcr(16, 256, 0, 1e-10, 0.0, eta)
    assert ifail == 0 and rho <= 1e-10 * np.linalg.norm(eta)


def test_unsafe_even_sw_term_leaves_sap_gcr_alone(setup):
    """an unsafe even-site block does not concern the eo block solver, which
    inverts the odd sites only (sap_gcr.c:180-196)"""
    vol = setup.vol
    eta = setup.source(6)
    qb.set_sap_parms(BS, 1, 4, 5)
    try:
        flag = qb.upload_swd(_unsafe(setup.swd, vol, 9))               # an even site
        assert flag & 1 and not flag & 2
        psi, rho, ifail, st = qb.sap_gcr(16, 256, 0, 1e-10, 0.0, eta)
        assert ifail != -3
    finally:
        assert qb.upload_swd(setup.swd) == 0
