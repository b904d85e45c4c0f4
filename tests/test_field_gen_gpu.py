"""The device's test-field generator against the reference's.

The reference makes its test gauge fields as U = expXsu3(eps, X) with X drawn
by random_alg (modules/linalg/liealg.c:289, a distribution proportional to
exp{tr X^2} in openQCD's su(3) convention), then applies the boundary
conditions.  The library's generator (b200_random_ud) uses its own Philox
numbers and its own SU(3) exponential, so the fields differ link by link;
what must agree is the distribution, which sets the roughness of every field
the benchmarks and solver tests run on.  Compared here on 16^4 at eps = 0.3
and 0.4, over the spatial links (the time links at x0 = N0-1 carry the
boundary sign):

- the mean and the variance of Re tr U / 3 and of |tr U|^2 / 9, within five
  standard errors of the difference of two independent sample means;
- the mean plaquette of the whole field (device plaquette sum against the
  reference's plaq_sum_dble), within 0.3 % (each is an average over 393,216
  plaquettes; the two normalisations of X that differ by a factor of two
  would move it by about 10 %).
"""
import numpy as np
import pytest

import openqcd_b200 as qb
import reflib

pytestmark = pytest.mark.gpu

L = (16, 16, 16, 16)


@pytest.fixture(scope="module")
def ref():
    if not reflib.ensure_built(L, portable=True):
        pytest.skip("reference oracle for 16^4 is not built")
    r = reflib.RefLib(L, portable=True)
    r.init(bc=3, seed=99, csw=1.7, m0=-0.05, eoflg=0)
    return r


def _spatial_traces(ud):
    """Re tr U / 3 and |tr U|^2 / 9 of the spatial links in the reference's
    8-links-per-odd-site array (slots 2 mu, 2 mu + 1 hold direction mu)"""
    u = ud.reshape(-1, 8, 9, 2)[:, 2:, :, :].reshape(-1, 9, 2)
    tr_re = u[:, 0, 0] + u[:, 4, 0] + u[:, 8, 0]
    tr_im = u[:, 0, 1] + u[:, 4, 1] + u[:, 8, 1]
    return tr_re / 3.0, (tr_re ** 2 + tr_im ** 2) / 9.0


def _close(a, b, k=5.0):
    se = np.sqrt(a.var() / a.size + b.var() / b.size)
    return abs(a.mean() - b.mean()) <= k * se, a.mean(), b.mean(), se


@pytest.mark.parametrize("eps", [0.3, 0.4])
def test_link_distribution(ref, eps):
    ref.gen_links(eps, 1357)
    ud_ref = ref.ud()
    qb.geometry(L, (4, 4, 4, 4), ref.ipt())
    qb.set_parms(1.7, -0.05, 0)
    qb.random_ud(eps, 2468)
    ud_dev = qb.download_ud(ref.vol)
    for a, b in zip(_spatial_traces(ud_dev), _spatial_traces(ud_ref)):
        ok, ma, mb, se = _close(a, b)
        assert ok, "eps %g: device mean %.6f, reference mean %.6f, se %.2e" % (eps, ma, mb, se)
        assert abs(a.var() / b.var() - 1.0) < 0.03, (a.var(), b.var())


@pytest.mark.parametrize("eps", [0.3])
def test_mean_plaquette(ref, eps):
    ref.gen_links(eps, 97531)
    p_ref = ref.plaq_sum()
    qb.geometry(L, (4, 4, 4, 4), ref.ipt())
    qb.set_parms(1.7, -0.05, 0)
    qb.random_ud(eps, 86420)
    p_dev = qb.plaq_sum()
    n = 6 * ref.vol
    assert abs(p_dev / p_ref - 1.0) < 3e-3, (p_dev / (3 * n), p_ref / (3 * n))
