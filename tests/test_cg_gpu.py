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


# ------------------------------------------------------------ multi-shift CG
def normal_eo(setup, mu, psi):
    """(Dwhat(mu)^dag Dwhat(mu) psi) on the even sites, with the reference
    (whose Dwhat_dble needs the odd SW term inverted)"""
    setup.ref.sw_term(2)
    out = g5(setup.ref.dirac_dble(5, -mu, g5(setup.ref.dirac_dble(5, mu, psi))))
    setup.ref.sw_term(0)
    return out


def run_tmcgm(setup, nmx, istop, res, mus, eta):
    setup.ref.sw_term(2)                  # tmcgm needs the odd SW term inverted
    out_r = setup.ref.tmcgm(nmx, istop, res, mus, eta)
    setup.ref.sw_term(0)
    return out_r, qb.tmcgm(nmx, istop, res, mus, eta)


@pytest.mark.parametrize("istop", [0, 1])
def test_tmcgm(setup, istop):
    """mscg.c with tmcgm's operator pair: FP64 iterations like the
    reference's, so solutions agree to 1e-9 and the total iteration count
    (including the final residual checks) to within two."""
    mus = [0.05, 0.0, 0.2, 0.1]
    res = [1e-10, 1e-9, 1e-8, 1e-10]
    eta = setup.source(31)
    n = setup.vol // 2 * 24
    (psr, fr, sr), (ps, f, s) = run_tmcgm(setup, 2000, istop, res, mus, eta)
    assert f == fr == 0
    assert abs(s - sr) <= 2, (s, sr)
    for k, mu in enumerate(mus):
        assert rel_norm_err(ps[k][:n], psr[k][:n]) <= 1e-9, (k, rel_norm_err(ps[k][:n], psr[k][:n]))
        assert not ps[k][n:].any()
        if istop == 0:
            r = eta[:n] - normal_eo(setup, mu, ps[k])[:n]
            assert np.linalg.norm(r) / np.linalg.norm(eta[:n]) <= 1.05 * res[k]


def test_tmcgm_many_shifts(setup):
    """14 shifts: more than one group of shifted systems per update launch"""
    mus = [0.01 * k for k in range(14)][::-1]
    res = [1e-9] * 14
    eta = setup.source(32)
    n = setup.vol // 2 * 24
    (psr, fr, sr), (ps, f, s) = run_tmcgm(setup, 3000, 0, res, mus, eta)
    assert f == fr == 0
    assert abs(s - sr) <= 2, (s, sr)
    for k in range(14):
        assert rel_norm_err(ps[k][:n], psr[k][:n]) <= 1e-8


def test_tmcgm_single_and_limits(setup):
    """one shift; too few iterations (ifail -1, status nmx); zero source"""
    eta = setup.source(33)
    n = setup.vol // 2 * 24
    (psr, fr, sr), (ps, f, s) = run_tmcgm(setup, 2000, 0, [1e-10], [0.03], eta)
    assert f == fr == 0 and abs(s - sr) <= 2
    assert rel_norm_err(ps[0][:n], psr[0][:n]) <= 1e-9
    (psr, fr, sr), (ps, f, s) = run_tmcgm(setup, 10, 0, [1e-10, 1e-10], [0.0, 0.1], eta)
    assert f == fr == -1 and s == sr == 10
    zero = np.zeros_like(eta)
    ps, f, s = qb.tmcgm(100, 0, [1e-10, 1e-10], [0.0, 0.1], zero)
    assert f == 0 and s == 0 and not any(p.any() for p in ps)


def test_tmcgm_bad_residue(setup):
    eta = setup.source(34)
    with pytest.raises(qb.B200Error, match="residues"):
        qb.tmcgm(100, 0, [1e-10, 0.0], [0.0, 0.1], eta)
