"""CG on the normal equations (modules/linsolv/cgne.c with the drivers
tmcg/tmcgeo of modules/forces/tmcg.c) against the reference on the same
fields: FP64 residual |eta - Dw^dag Dw psi|/|eta| <= 1.5 res (checked with
the reference's Dw_dble), solution within 1e-8 of the reference's, and the
iteration count within two of the reference's (the FP32 inner products sum
in another order)."""
import numpy as np
import pytest

import openqcd_b200 as qb
from helpers import Setup, rel_norm_err

pytestmark = pytest.mark.gpu

L = (8, 8, 8, 8)


@pytest.fixture(scope="module")
def setup():
    return Setup(L, (4, 4, 4, 4), eps=0.4, csw=1.5, m0=-0.1)


def g5(x):
    y = np.array(x, dtype=np.float64).reshape(-1, 24)
    y[:, 12:] *= -1.0
    return y.reshape(-1)


def normal_op(setup, mu, psi):
    """Dw(mu)^dag Dw(mu) psi = g5 Dw(-mu) g5 Dw(mu) psi with the reference."""
    return g5(setup.ref.dirac_dble(0, -mu, g5(setup.ref.dirac_dble(0, mu, psi))))


@pytest.mark.parametrize("mu", [0.0, 0.05])
def test_tmcg(setup, mu):
    eta = setup.source(21)
    res = 1e-10
    psi_r, rho_r, f_r, st_r = setup.ref.tmcg(2000, 0, res, mu, eta)
    psi, rho, f, st = qb.tmcg(2000, 0, res, mu, eta)
    assert f == f_r == 0
    assert abs(st - st_r) <= 2, (st, st_r)
    r = eta - normal_op(setup, mu, psi)
    assert np.linalg.norm(r) / np.linalg.norm(eta) <= 1.5 * res
    assert rel_norm_err(psi, psi_r) <= 1e-8


def test_tmcgeo(setup):
    """Even sites only: Dwhat^dag Dwhat psi_e = eta_e."""
    mu = 0.02
    eta = setup.source(22)
    n = setup.vol // 2 * 24
    setup.ref.sw_term(2)                  # the reference needs the odd SW term inverted
    psi_r, rho_r, f_r, st_r = setup.ref.tmcg(2000, 0, 1e-10, mu, eta, eo=True)
    setup.ref.sw_term(0)
    psi, rho, f, st = qb.tmcg(2000, 0, 1e-10, mu, eta, eo=True)
    assert f == f_r == 0
    assert abs(st - st_r) <= 2, (st, st_r)
    assert rel_norm_err(psi[:n], psi_r[:n]) <= 1e-8


def test_tmcg_zero_source(setup):
    eta = np.zeros(setup.vol * 24)
    psi, rho, f, st = qb.tmcg(100, 0, 1e-10, 0.0, eta)
    assert rho == 0.0 and f == 0 and not psi.any()
