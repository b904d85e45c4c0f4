"""Exponential SW term (isw = 1: c exp{[csw/(4+m0)] (i/4) sigma F},
modules/sw_term/sw_term.c:46-49 with the exponential of swexp.c:239) built
on the device from the links, against a private instance of the reference
run with the same SW type: the matrices and their inverses (1/c) exp(-A) to
1e-14 per site, the Dirac operators that use them to 1e-13."""
import numpy as np
import pytest

import openqcd_b200 as qb
from helpers import OPS, Setup, site_rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    s = Setup((8, 8, 8, 8), (4, 4, 4, 4), eps=0.4, csw=1.7, m0=-0.1, isw=1)
    qb.upload_ud(s.ud)
    assert qb.sw_term() == 0          # the device builds its own exponential SW term
    yield s
    qb.set_parms(1.5, 0.0, 0, isw=0)


def pauli_rel_err(a, b):
    a = np.asarray(a).reshape(-1, 36)
    b = np.asarray(b).reshape(-1, 36)
    return float((np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)).max())


def test_swexp_matrices(setup):
    dev = qb.download_swd(setup.vol, 0)
    assert pauli_rel_err(dev, setup.swd) <= 1e-14


def test_swexp_inverse(setup):
    setup.ref.sw_term(3)              # ALL_PTS: the reference's (1/c) exp(-A)
    ref_inv = setup.ref.swd()
    setup.ref.sw_term(0)
    dev_inv = qb.download_swd(setup.vol, 1)
    assert pauli_rel_err(dev_inv, ref_inv) <= 1e-14


@pytest.mark.parametrize("op", OPS)
def test_swexp_dirac_dble(setup, op):
    s = setup.source(41)
    r0 = setup.source(42)
    mu = 0.07
    if op == "Dwhat":
        setup.ref.sw_term(2)
    ref = setup.ref.dirac_dble(OPS.index(op), mu, s, r0)
    if op == "Dwhat":
        setup.ref.sw_term(0)
    out = qb.dirac_ref(op, 64, mu, s, r0)
    assert site_rel_err(out, ref, setup.vol) <= 1e-13


def test_sw_type_range(setup):
    with pytest.raises(qb.B200Error, match="isw"):
        qb.check(qb.lib().b200_set_sw_type(2))


def test_swexp_dfl_modes(setup):
    """Subspace generation shifts the bare mass; with the exponential form
    the SW field is rebuilt from the links at the generation mass and again
    at the end (the mass sits in the exponent): the field afterwards is the
    one before, and the deflated solver converges on the same operator."""
    before = qb.download_swd(setup.vol, 0)
    qb.set_sap_parms((4, 4, 4, 4), 1, 4, 5)
    qb.set_dfl_parms((4, 4, 4, 4), 8)
    qb.set_dfl_pro_parms(16, 256, 1e-2, 24, 1e-2)
    qb.set_dfl_gen_parms(1.0 / (2.0 * (4.0 - 0.1)), 0.0, 6, 4, 4)
    ifail, st = qb.dfl_modes(3)
    assert ifail == 0
    after = qb.download_swd(setup.vol, 0)
    assert pauli_rel_err(after, before) <= 1e-15
    eta = setup.source(43)
    psi, rho, ifail, st = qb.dfl_sap_gcr(16, 256, 0, 1e-10, 0.0, eta)
    assert ifail == 0
    r = eta - setup.ref.dirac_dble(0, 0.0, psi)
    assert np.linalg.norm(r) / np.linalg.norm(eta) <= 1.5e-10
