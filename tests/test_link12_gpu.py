"""12-real FP32 links (no reference counterpart): with b200_set_sap_link12
on (the default) the FP32 Dirac operators and the SAP solver read the first
two rows of each link and rebuild the third as conj(row1 x row2), negated on
the time links at x0 = N0-1 that carry the antiperiodic phase.  The results
agree with the 18-real reads to FP32 rounding and with the reference's FP32
operators (2e-6 per site); a field in which one link breaks the relation
with the sign its position implies is read in full, giving the 18-real
results bit for bit."""
import numpy as np
import pytest

import openqcd_b200 as qb
from helpers import OPS, Setup, site_rel_err

pytestmark = pytest.mark.gpu

L = (8, 8, 8, 8)
BS = (4, 4, 4, 4)
MU = 0.07


@pytest.fixture(scope="module")
def setup():
    s = Setup(L, BS, eps=0.4, csw=1.5, m0=-0.05)
    yield s
    qb.set_sap_link12(1)


def both(fn):
    out = []
    for on in (0, 1):
        qb.set_sap_link12(on)
        out.append(fn())
    qb.set_sap_link12(1)
    return out


@pytest.mark.parametrize("op", OPS)
def test_fp32_operators_link12(setup, op):
    s = setup.source(21)
    r0 = setup.source(22)
    r18, r12 = both(lambda: qb.dirac_ref(op, 32, MU, s, r0))
    assert site_rel_err(r12, r18, setup.vol) <= 1e-6
    if op == "Dwhat":
        setup.ref.sw_term(2)       # the reference's Dwhat needs the odd SW term inverted
    ref = setup.ref.dirac(OPS.index(op), MU, s, r0)
    if op == "Dwhat":
        setup.ref.sw_term(0)
    assert site_rel_err(r12, ref, setup.vol) <= 2e-6


def test_dirac_multi_link12(setup):
    """The residual-update form r = sub - Dw s of the deflated preconditioner."""
    S = qb.DevField(32)
    S.from_ref(setup.source(23).astype(np.float32))
    U = qb.DevField(32)
    U.from_ref(setup.source(24).astype(np.float32))

    def run():
        R = qb.DevField(32)
        qb.dev_dirac_multi(MU, [S], [R], [U])
        out = R.to_ref(setup.vol)
        R.free()
        return out

    r18, r12 = both(run)
    assert site_rel_err(r12, r18, setup.vol) <= 1e-6
    assert not np.array_equal(r12, r18)     # the 12-real reads were used
    assert qb.links12_active()


def test_sap_gcr_link12(setup):
    qb.set_sap_parms(BS, 1, 4, 5)
    eta = setup.source(25)
    (p18, _, f18, s18), (p12, _, f12, s12) = both(lambda: qb.sap_gcr(16, 256, 0, 1e-10, MU, eta))
    assert f18 == 0 and f12 == 0 and abs(s12 - s18) <= 1
    for psi in (p18, p12):
        r = eta - setup.ref.dirac_dble(0, MU, psi)
        assert np.linalg.norm(r) / np.linalg.norm(eta) <= 1.5e-10


def test_link12_check_rejects(setup):
    """One interior link multiplied by -1 (a U(3) matrix with det -1): the
    check fails and every read is the 18-real one."""
    ud = setup.ud.copy().reshape(setup.vol // 2, 8, 18)
    ud[5, 4] *= -1.0                      # direction 2, forward, at an interior site
    qb.upload_ud(ud.reshape(-1))
    try:
        s = setup.source(26)
        r18, r12 = both(lambda: qb.dirac_ref("Dw", 32, MU, s))
        assert np.array_equal(r12, r18)
        assert not qb.links12_active()
    finally:
        qb.upload_ud(setup.ud)
        qb.upload_swd(setup.swd)
