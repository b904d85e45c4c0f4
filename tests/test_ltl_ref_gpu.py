"""The reference's little solver restated on the device (modules/dfl/ltl_gcr.c
with linsolv/fgcr4vd.c, linsolv/gcr4v.c and the global-mode deflation of
little/ltl_modes.c), its pieces (the even-odd parts of the little operator,
the FP32 little operators, the little-little matrix and the projections),
against the reference on the same subspace: the reference's block basis and
its little modes are loaded into the device.  Bars: 1e-12 for FP64 pieces,
1e-5 for FP32 ones; the little solve agrees in its iteration counts and to
1e-4 in the solution (its inner solver is FP32); the deflated SAP+GCR with
this little solver to 1e-8 and one outer step."""
import numpy as np
import pytest

import openqcd_b200 as qb
from helpers import Setup, rel_norm_err

pytestmark = pytest.mark.gpu

L = (8, 8, 8, 8)
BS = (4, 4, 4, 4)
NS = 8
M0 = -0.2
KAPPA = 1.0 / (2.0 * (4.0 + M0))
MU = 0.01


@pytest.fixture(scope="module")
def setup():
    s = Setup(L, BS, eps=0.4, csw=1.5, m0=M0)
    s.ref.set_sap_parms(BS, 1, 4, 5)
    s.nv = s.ref.dfl_init(BS, NS, nkv=16, nmx=256, res=1e-2, nmx_gcr=24, res_gcr=1e-2, kappa=KAPPA, mu=0.0,
                          ninv=5, nmr=4, ncy=4)
    f, st = s.ref.dfl_modes(7)
    assert f == 0
    qb.set_sap_parms(BS, 1, 4, 5)
    assert qb.set_dfl_parms(BS, NS) == s.nv
    qb.set_dfl_pro_parms(16, 256, 1e-2, 24, 1e-2)
    qb.set_dfl_gen_parms(KAPPA, 0.0, 5, 4, 4)
    for l in range(NS):
        qb.dfl_set_basis(l, s.ref.dfl_get_basis(l))
    for l in range(NS):
        qb.dfl_set_lmode(l, s.ref.dfl_get_lmode(l, s.nv))
    s.rng = np.random.default_rng(17)
    yield s
    qb.set_ltl_solver(0)


def rvec(s, dtype=np.float64):
    return s.rng.standard_normal(2 * s.nv).astype(dtype)


@pytest.mark.parametrize("name", ["Aweeinv_dble", "Awooinv_dble", "Awoe_dble", "Aweo_dble"])
def test_little_eo_pieces(setup, name):
    v, w0 = rvec(setup), rvec(setup)
    ref, f = setup.ref.little(qb.LITTLE_EO[name], MU, v, w0)
    dev, g = qb.little_eo(name, MU, v, w0)
    assert f == g == 0
    assert rel_norm_err(dev, ref) <= 1e-12


@pytest.mark.parametrize("which", [0, 1, 2, 3, 4, 5], ids=["Aw", "Awhat", "Aweeinv", "Awooinv", "Awoe", "Aweo"])
def test_little_fp32(setup, which):
    v, w0 = rvec(setup, np.float32), rvec(setup, np.float32)
    ref = setup.ref.little32(which, MU, v, w0)
    dev = qb.little32(which, MU, v, w0)
    assert rel_norm_err(dev.astype(np.float64), ref.astype(np.float64)) <= 1e-5


def test_ltl_modes_and_projections(setup):
    mref, f = setup.ref.ltl_modes(MU, NS)
    qb.little(1, MU, rvec(setup))          # set_Awhat(MU) on the device
    assert f == 0 and qb.set_ltl_modes() == 0
    m = qb.ltl_matrix(NS)
    assert rel_norm_err(m, mref) <= 1e-10
    for which in (0, 1, 2):
        v, w = rvec(setup), rvec(setup)
        rv, rw = setup.ref.dfl_proj(which, v, w)
        dv, dw = qb.dfl_proj(which, v, w)
        assert rel_norm_err(dv, rv) <= 1e-11, which
        if which:
            assert rel_norm_err(dw, rw) <= 1e-11, which
    v = rvec(setup, np.float32)
    assert rel_norm_err(qb.dfl_Lv(v).astype(np.float64), setup.ref.dfl_Lv(v).astype(np.float64)) <= 2e-5


@pytest.mark.parametrize("mu", [0.0, 0.05])
def test_ltl_gcr_reference_algorithm(setup, mu):
    eta = rvec(setup)
    psi_r, rho_r, f_r, st_r = setup.ref.ltl_gcr(mu, eta)
    prev = qb.set_ltl_solver(1)
    try:
        psi, rho, f, st = qb.ltl_gcr(mu, eta)
    finally:
        qb.set_ltl_solver(prev)
    assert f == f_r == 0
    assert abs(st[0] - st_r[0]) <= 1, (st, st_r)
    assert abs(st[1] - st_r[1]) <= 3, (st, st_r)
    assert st[1] > 0
    assert rel_norm_err(psi, psi_r) <= 1e-4
    assert abs(rho - rho_r) <= 1e-3 * rho_r + 1e-14


def test_dfl_sap_gcr_with_reference_little_solver(setup):
    eta = setup.source(31)
    psi_r, rho_r, f_r, st_r = setup.ref.dfl_sap_gcr(16, 256, 0, 1e-10, 0.0, eta)
    prev = qb.set_ltl_solver(1)
    try:
        psi, rho, f, st = qb.dfl_sap_gcr(16, 256, 0, 1e-10, 0.0, eta)
    finally:
        qb.set_ltl_solver(prev)
    assert f == f_r == 0
    # outer GCR steps, average fgcr4vd and gcr4v Krylov vectors per little solve
    for k in range(3):
        assert abs(st[k] - st_r[k]) <= 1, (st, st_r)
    assert st[2] > 0
    assert rel_norm_err(psi, psi_r) <= 1e-8
    r = eta - setup.ref.dirac_dble(0, 0.0, psi)
    assert np.linalg.norm(r) / np.linalg.norm(eta) <= 1.5e-10
