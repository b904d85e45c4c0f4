"""Block size 6^4 (648 sites per parity, the SAP/DFL block of the 48^3x96
deflated solve) on a 12^4 lattice: the Dirac operators, SAP cycles, SAP+GCR
and the deflation pieces against the reference built with the same block
size (oracle/_ref/12x12x12x12_t4_c, plain-C code paths so that SAP agrees to
FP32 rounding).  Bars as in the 4^4 tests: 1e-13 per site for FP64
operators, 2e-6 for FP32 ones, 1e-5 for SAP cycles, FP64 true residual for
the solvers."""
import numpy as np
import pytest

import openqcd_b200 as qb
from helpers import OPS, Setup, rel_norm_err, site_rel_err

pytestmark = pytest.mark.gpu

L = (12, 12, 12, 12)
BS = (6, 6, 6, 6)
NS = 8
M0 = -0.2


@pytest.fixture(scope="module")
def setup():
    s = Setup(L, BS, eps=0.4, csw=1.5, m0=M0, portable=True)
    s.ref.set_sap_parms(BS, 1, 4, 5)
    qb.set_sap_parms(BS, 1, 4, 5)
    return s


@pytest.mark.parametrize("op", OPS)
def test_dirac_dble(setup, op):
    s = setup.source(21)
    r0 = setup.source(22)
    mu = 0.03
    if op == "Dwhat":
        setup.ref.sw_term(2)       # reference needs the odd SW term inverted
    ref = setup.ref.dirac_dble(OPS.index(op), mu, s, r0)
    if op == "Dwhat":
        setup.ref.sw_term(0)
    out = qb.dirac_ref(op, 64, mu, s, r0)
    assert site_rel_err(out, ref, setup.vol) <= 1e-13


@pytest.mark.parametrize("op", OPS)
def test_staged_equals_direct(setup, op):
    """The FP64 operators with bulk-staged SW matrices (648-site chunks:
    five tiles of 128 sites and a partial one) against the direct-read
    kernel: the same arithmetic."""
    s = setup.source(13)
    r0 = setup.source(14)
    prev = qb.set_dw_staged(0)
    try:
        out = []
        for mode in (0, 1):
            qb.set_dw_staged(mode)
            out.append(qb.dirac_ref(op, 64, 0.137, s, r0))
    finally:
        qb.set_dw_staged(prev)
    assert site_rel_err(out[1], out[0], setup.vol) <= 1e-15


@pytest.mark.parametrize("op", ["Dw", "Dwhat"])
def test_dirac_fp32(setup, op):
    s = setup.source(23).astype(np.float32)
    if op == "Dwhat":
        setup.ref.sw_term(2)
    ref = setup.ref.dirac(OPS.index(op), 0.03, s)
    if op == "Dwhat":
        setup.ref.sw_term(0)
    out = qb.dirac_ref(op, 32, 0.03, s)
    assert site_rel_err(out, ref, setup.vol) <= 2e-6


@pytest.mark.parametrize("isolv", [1, 0])
def test_sap_cycles(setup, isolv):
    eta = setup.source(24).astype(np.float32)
    psi0 = np.zeros_like(eta)
    ncy = 3
    setup.ref.set_sap_parms(BS, isolv, 4, ncy)
    psi_ref, rho_ref, f = setup.ref.sap(0.02, isolv, 4, ncy, psi0, eta)
    assert f == 0
    psi, rho = psi0, eta
    for _ in range(ncy):
        psi, rho = qb.sap_ref(0.02, isolv, 4, psi, rho)
    setup.ref.set_sap_parms(BS, 1, 4, 5)
    assert rel_norm_err(psi, psi_ref) <= 1e-5
    assert rel_norm_err(rho, rho_ref) <= 1e-5


def test_sap_gcr(setup):
    eta = setup.source(25)
    qb.set_sap_parms(BS, 1, 4, 5)
    psi_ref, _, ifail_ref, st_ref = setup.ref.sap_gcr(16, 256, 0, 1e-10, 0.0, eta)
    psi, rho, ifail, st = qb.sap_gcr(16, 256, 0, 1e-10, 0.0, eta)
    assert ifail == ifail_ref == 0
    assert abs(st - st_ref) <= 1
    r = eta - setup.ref.dirac_dble(0, 0.0, psi)
    assert np.linalg.norm(r) / np.linalg.norm(eta) <= 1.5e-10


@pytest.fixture(scope="module")
def dfl(setup):
    s = setup
    s.nv = s.ref.dfl_init(BS, NS, kappa=1.0 / (2.0 * (4.0 + M0)), ninv=5, nmr=4, ncy=4)
    f, _ = s.ref.dfl_modes(7)
    assert f == 0
    s.basis = [s.ref.dfl_get_basis(l) for l in range(NS)]
    assert qb.set_dfl_parms(BS, NS) == s.nv
    qb.set_dfl_pro_parms(16, 256, 1e-2, 24, 1e-2)
    qb.set_dfl_gen_parms(1.0 / (2.0 * (4.0 + M0)), 0.0, 5, 4, 4)
    for l in range(NS):
        qb.dfl_set_basis(l, s.basis[l])
    return s


def test_dfl_s2vd_Aw(dfl):
    s = np.random.default_rng(7).standard_normal(dfl.vol * 24).astype(np.float32)
    vd_ref = dfl.ref.dfl_s2vd(s)
    vd = qb.dfl_s2vd(s, dfl.nv)
    assert np.abs(vd - vd_ref).max() <= 2e-6 * np.abs(vd_ref).max()
    v = np.random.default_rng(8).standard_normal(2 * dfl.nv)
    assert rel_norm_err(qb.little(0, 0.01, v)[0], dfl.ref.little(0, 0.01, v)[0]) <= 1e-10
    assert rel_norm_err(qb.little(1, 0.01, v)[0], dfl.ref.little(1, 0.01, v)[0]) <= 1e-10


def test_dfl_sap_gcr(dfl):
    eta = dfl.source(26)
    psi_ref, _, ifail_ref, st_ref = dfl.ref.dfl_sap_gcr(16, 256, 0, 1e-10, 0.0, eta)
    psi, rho, ifail, st = qb.dfl_sap_gcr(16, 256, 0, 1e-10, 0.0, eta)
    assert ifail == ifail_ref == 0
    assert abs(st[0] - st_ref[0]) <= max(2, st_ref[0] // 5), (st, st_ref)
    r = eta - dfl.ref.dirac_dble(0, 0.0, psi)
    assert np.linalg.norm(r) / np.linalg.norm(eta) <= 1.5e-10


def test_dfl_modes_device(dfl):
    eta = dfl.source(27)
    _, _, _, st_ref = dfl.ref.dfl_sap_gcr(16, 256, 0, 1e-10, 0.0, eta)
    ifail, st = qb.dfl_modes(5)
    assert ifail == 0
    psi, rho, ifail, st = qb.dfl_sap_gcr(16, 256, 0, 1e-10, 0.0, eta)
    assert ifail == 0 and st[0] <= st_ref[0] + max(3, st_ref[0] // 4), (st, st_ref)
    r = eta - dfl.ref.dirac_dble(0, 0.0, psi)
    assert np.linalg.norm(r) / np.linalg.norm(eta) <= 1.5e-10
