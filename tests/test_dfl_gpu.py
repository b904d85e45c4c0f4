"""Parity of the device deflation with the reference (modules/dfl/,
modules/little/).

The block basis is taken from the reference (its dfl_modes run on the CPU)
and loaded into the device library, so that restriction, prolongation and
the little Dirac operator can be compared entry by entry:

* dfl_s2vd / dfl_vd2s (dfl_subspace.c:83, :126) work in FP32 with
  single-precision results: 2e-6 relative to the largest component;
* Aw_dble and Awhat_dble (Aw_dble.c:122, :361) are built in FP64 from the
  same FP32 basis: 1e-10 relative;
* ltl_gcr (ltl_gcr.c:155) is checked against a dense solve of the little
  system assembled column by column from the device Aw_dble;
* dfl_sap_gcr (dfl_sap_gcr.c:353) reaches the FP64 true residual computed by
  the reference's Dw_dble, in an iteration count close to the reference's;
* dfl_modes on the device (own random fields) generates a subspace with
  which the deflated solver converges as fast as with the reference's.
"""
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


@pytest.fixture(scope="module")
def setup():
    s = Setup(L, BS, eps=0.4, csw=1.5, m0=M0)
    s.ref.set_sap_parms(BS, 1, 4, 5)
    s.nv = s.ref.dfl_init(BS, NS, nkv=16, nmx=256, res=1e-2, nmx_gcr=24, res_gcr=1e-2, kappa=KAPPA, mu=0.0,
                          ninv=5, nmr=4, ncy=4)
    f, st = s.ref.dfl_modes(7)
    assert f == 0
    s.basis = [s.ref.dfl_get_basis(l) for l in range(NS)]
    qb.set_sap_parms(BS, 1, 4, 5)
    assert qb.set_dfl_parms(BS, NS) == s.nv
    qb.set_dfl_pro_parms(16, 256, 1e-2, 24, 1e-2)
    qb.set_dfl_gen_parms(KAPPA, 0.0, 5, 4, 4)
    return s


def load_reference_basis(s):
    for l in range(NS):
        qb.dfl_set_basis(l, s.basis[l])


def cplx(v):
    return np.asarray(v, dtype=np.float64).view(np.complex128)


def test_basis_round_trip(setup):
    load_reference_basis(setup)
    for l in (0, NS - 1):
        assert np.array_equal(qb.dfl_get_basis(l, setup.vol), setup.basis[l])


def test_s2vd(setup):
    load_reference_basis(setup)
    s = np.random.default_rng(1).standard_normal(setup.vol * 24).astype(np.float32)
    vd_ref = setup.ref.dfl_s2vd(s)
    vd = qb.dfl_s2vd(s, setup.nv)
    assert np.abs(vd - vd_ref).max() <= 2e-6 * np.abs(vd_ref).max()


def test_vd2s(setup):
    load_reference_basis(setup)
    vd = np.random.default_rng(2).standard_normal(2 * setup.nv)
    s_ref = setup.ref.dfl_vd2s(vd)
    s = qb.dfl_vd2s(vd, setup.vol)
    assert np.abs(s - s_ref).max() <= 2e-6 * np.abs(s_ref).max()


def test_projector(setup):
    """dfl_s2vd(dfl_vd2s(v)) = v for an orthonormal block basis."""
    load_reference_basis(setup)
    vd = np.random.default_rng(3).standard_normal(2 * setup.nv)
    back = qb.dfl_s2vd(qb.dfl_vd2s(vd, setup.vol), setup.nv)
    assert np.abs(back - vd).max() <= 1e-5 * np.abs(vd).max()


@pytest.mark.parametrize("mu", [0.0, 0.05])
def test_Aw_dble(setup, mu):
    load_reference_basis(setup)
    v = np.random.default_rng(4).standard_normal(2 * setup.nv)
    w_ref, _ = setup.ref.little(0, mu, v)
    w, _ = qb.little(0, mu, v)
    assert rel_norm_err(w, w_ref) <= 1e-10


@pytest.mark.parametrize("mu", [0.0, 0.05])
def test_Awhat_dble(setup, mu):
    load_reference_basis(setup)
    rng = np.random.default_rng(5)
    v = rng.standard_normal(2 * setup.nv)
    w0 = rng.standard_normal(2 * setup.nv)
    w_ref, f_ref = setup.ref.little(1, mu, v, w0)
    w, f = qb.little(1, mu, v, w0)
    assert f == f_ref == 0
    assert rel_norm_err(w, w_ref) <= 1e-10
    # the odd half of w is left unchanged
    assert np.array_equal(w[setup.nv:], w0[setup.nv:])


def test_ltl_gcr_dense(setup):
    load_reference_basis(setup)
    nv, mu = setup.nv, 0.01
    A = np.zeros((nv, nv), dtype=np.complex128)
    e = np.zeros(2 * nv)
    for j in range(nv):
        e[:] = 0.0
        e[2 * j] = 1.0
        A[:, j] = cplx(qb.little(0, mu, e)[0])
    eta = np.random.default_rng(6).standard_normal(2 * nv)
    x = np.linalg.solve(A, cplx(eta))
    qb.set_dfl_pro_parms(16, 256, 1e-12, 24, 1e-2)
    try:
        psi, rho, ifail, st = qb.ltl_gcr(mu, eta)
    finally:
        qb.set_dfl_pro_parms(16, 256, 1e-2, 24, 1e-2)
    assert ifail == 0 and st[0] > 0
    assert np.linalg.norm(cplx(psi) - x) <= 1e-9 * np.linalg.norm(x)
    # the reference to its default accuracy (res = 1e-2)
    psi_ref, rho_ref, ifail_ref, _ = setup.ref.ltl_gcr(mu, eta)
    assert ifail_ref == 0
    assert np.linalg.norm(cplx(psi_ref) - x) <= 0.1 * np.linalg.norm(x)


@pytest.mark.parametrize("mu", [0.0, 0.02])
def test_dfl_sap_gcr_reference_basis(setup, mu):
    load_reference_basis(setup)
    eta = setup.source(11)
    nkv, nmx, res = 16, 256, 1e-10
    psi_ref, rho_ref, ifail_ref, st_ref = setup.ref.dfl_sap_gcr(nkv, nmx, 0, res, mu, eta)
    psi, rho, ifail, st = qb.dfl_sap_gcr(nkv, nmx, 0, res, mu, eta)
    assert ifail_ref == 0 and ifail == 0
    assert abs(st[0] - st_ref[0]) <= max(2, st_ref[0] // 5), (st, st_ref)
    r = eta - setup.ref.dirac_dble(0, mu, psi)
    true_res = np.linalg.norm(r) / np.linalg.norm(eta)
    assert true_res <= 1.5 * res, true_res
    assert rho <= res * np.linalg.norm(eta) * 1.00001
    assert rel_norm_err(psi, psi_ref) <= 1e-8


def test_dfl_sap_gcr_in_place_zero_source(setup):
    load_reference_basis(setup)
    eta = np.zeros(setup.vol * 24)
    psi, rho, ifail, st = qb.dfl_sap_gcr(16, 64, 0, 1e-8, 0.0, eta)
    assert ifail == 0 and rho == 0.0 and not psi.any()


def test_dfl_modes_device(setup):
    """Subspace generated on the device: orthonormal block basis, and the
    deflated solver converges as fast as with the reference's subspace."""
    eta = setup.source(12)
    _, _, ifail_ref, st_ref = setup.ref.dfl_sap_gcr(16, 256, 0, 1e-10, 0.0, eta)
    ifail, st = qb.dfl_modes(3)
    assert ifail == 0
    # the parameters of the solve are restored
    b0 = qb.dfl_get_basis(0, setup.vol).astype(np.float64)
    assert abs(np.dot(b0, b0) - setup.vol // (BS[0] * BS[1] * BS[2] * BS[3])) < 1e-3 * np.dot(b0, b0)
    psi, rho, ifail, st = qb.dfl_sap_gcr(16, 256, 0, 1e-10, 0.0, eta)
    assert ifail == 0
    assert st[0] <= st_ref[0] + max(3, st_ref[0] // 4), (st, st_ref)
    r = eta - setup.ref.dirac_dble(0, 0.0, psi)
    assert np.linalg.norm(r) / np.linalg.norm(eta) <= 1.5e-10
    # the SW term is back at the solver mass
    r2 = eta - qb.dirac_ref("Dw", 64, 0.0, psi)
    assert np.linalg.norm(r2 - r) <= 1e-12 * np.linalg.norm(eta)


def test_dfl_sap_gcr2(setup):
    load_reference_basis(setup)
    eta = setup.source(13)
    psi, rho, ifail, st = qb.dfl_sap_gcr2(16, 256, 0, 1e-10, 0.0, eta)
    assert ifail == [0, 0] and st[3:] == [0, 0, 0]
    r = eta - setup.ref.dirac_dble(0, 0.0, psi)
    assert np.linalg.norm(r) / np.linalg.norm(eta) <= 1.5e-10


def test_dfl_errors(setup):
    with pytest.raises(qb.B200Error):
        qb.set_dfl_parms((8, 4, 4, 4), NS)
    with pytest.raises(qb.B200Error):
        qb.set_dfl_parms(BS, 7)


@pytest.mark.parametrize("spread", [1.0, 1e-2])
def test_dfl_subspace_cholesky_qr(setup, spread):
    """dfl_subspace on the same FP32 modes as the reference's block
    Gram-Schmidt (dfl_subspace.c:171): the device's Cholesky QR gives the
    same Q to FP32 rounding, for Gaussian modes and for modes that are
    nearly parallel (a common field plus 1 % of noise, block condition
    numbers ~1e2)."""
    base = setup.source(90)
    modes = [((1.0 - spread) * base + spread * setup.source(91 + l)).astype(np.float32) for l in range(NS)]
    tol = 2e-6 if spread == 1.0 else 1e-4
    try:
        setup.ref.dfl_subspace(modes)
        ref = [setup.ref.dfl_get_basis(l) for l in range(NS)]
        qb.dfl_subspace(modes)
        dev = [qb.dfl_get_basis(l, setup.vol) for l in range(NS)]
        for l in range(NS):
            assert rel_norm_err(dev[l], ref[l]) <= tol, (l, rel_norm_err(dev[l], ref[l]))
    finally:
        setup.ref.dfl_subspace(setup.basis)
        load_reference_basis(setup)
