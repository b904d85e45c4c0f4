"""Non-cubic SAP blocks (8x4x4x4 and 4x4x8x4 on a 16^4 lattice): the device
layout tiles the lattice by the block, so the operators, the SAP cycle and
sap_gcr are compared with the reference (its plain-C build) for blocks that
are longer in one direction, with the bars of the cubic-block tests: 1e-13
per site for the FP64 operators, 2e-6 for FP32, 1e-5 for the SAP fields,
sap_gcr within one step and 1e-8 of the reference's solution."""
import numpy as np
import pytest

import openqcd_b200 as qb
from helpers import Setup, rel_norm_err, site_rel_err

pytestmark = pytest.mark.gpu

L = (16, 16, 16, 16)
MU = 0.03


@pytest.fixture(scope="module", params=[(8, 4, 4, 4), (4, 4, 8, 4)], ids=["8x4x4x4", "4x4x8x4"])
def setup(request):
    bs = request.param
    s = Setup(L, bs, eps=0.4, csw=1.5, m0=-0.05, portable=True, private=True)
    s.ref.set_sap_parms(bs, 1, 4, 2)
    qb.set_sap_parms(bs, 1, 4, 2)
    return s


@pytest.mark.parametrize("op", ["Dw", "Dwhat"])
def test_operators(setup, op):
    k = 0 if op == "Dw" else 5
    s = setup.source(31)
    if op == "Dwhat":
        setup.ref.sw_term(2)       # the reference's Dwhat needs the odd SW term inverted
    r64 = setup.ref.dirac_dble(k, MU, s)
    r32 = setup.ref.dirac(k, MU, s)
    if op == "Dwhat":
        setup.ref.sw_term(0)
    assert site_rel_err(qb.dirac_ref(op, 64, MU, s), r64, setup.vol) <= 1e-13
    assert site_rel_err(qb.dirac_ref(op, 32, MU, s), r32, setup.vol) <= 2e-6


@pytest.mark.parametrize("isolv", [1, 0])
def test_sap_cycles(setup, isolv):
    eta = setup.source(32).astype(np.float32)
    psi0 = np.zeros_like(eta)
    psi_ref, rho_ref, f = setup.ref.sap(MU, isolv, 4, 2, psi0, eta)
    assert f == 0
    psi, rho = psi0, eta
    for _ in range(2):
        psi, rho = qb.sap_ref(MU, isolv, 4, psi, rho)
    assert rel_norm_err(psi, psi_ref) <= 1e-5
    assert rel_norm_err(rho, rho_ref) <= 1e-5


def test_sap_gcr(setup):
    eta = setup.source(33)
    psi_ref, _, f_ref, st_ref = setup.ref.sap_gcr(16, 256, 0, 1e-10, MU, eta)
    psi, rho, f, st = qb.sap_gcr(16, 256, 0, 1e-10, MU, eta)
    assert f_ref == 0 and f == 0 and abs(st - st_ref) <= 1, (st, st_ref)
    r = eta - setup.ref.dirac_dble(0, MU, psi)
    assert np.linalg.norm(r) / np.linalg.norm(eta) <= 1.5e-10
    assert rel_norm_err(psi, psi_ref) <= 1e-8
