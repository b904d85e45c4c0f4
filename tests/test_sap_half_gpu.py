"""SAP on FP16 copies of the links and SW matrices (FP32 work vectors and
arithmetic; an option of this library with no reference counterpart).  It
is a preconditioner, so it is assessed by what the solver does with it: its
cycles stay within a few 1e-2 of the FP32 cycles of the reference
(modules/sap/sap.c:720) and of the identity rho = eta - Dw psi, and SAP+GCR
reaches the same FP64 true residual 1e-10, checked with the reference's
Dw_dble.  Measured on B200: one cycle is about 20 % faster at 6^4 blocks
(48^3x96), but GCR needs about 30 % more iterations, so the FP32 storage
stays the default; the bar below is 50 % more iterations.  Both block sizes
of the solver workloads (4^4 and 6^4) are covered."""
import numpy as np
import pytest

import openqcd_b200 as qb
from helpers import Setup, rel_norm_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=[((8, 8, 8, 8), (4, 4, 4, 4)), ((12, 12, 12, 12), (6, 6, 6, 6))],
                ids=["bs4", "bs6"])
def setup(request):
    L, bs = request.param
    s = Setup(L, bs, eps=0.4, csw=1.5, m0=-0.2, portable=True)
    s.ref.set_sap_parms(bs, 1, 4, 3)
    qb.set_sap_parms(bs, 1, 4, 3)
    yield s
    qb.set_sap_prec(32)


def test_half_cycles_close_to_reference(setup):
    eta = setup.source(31).astype(np.float32)
    psi0 = np.zeros_like(eta)
    psi_ref, rho_ref, f = setup.ref.sap(0.01, 1, 4, 3, psi0, eta)
    assert f == 0
    qb.set_sap_prec(16)
    try:
        psi, rho = psi0, eta
        for _ in range(3):
            psi, rho = qb.sap_ref(0.01, 1, 4, psi, rho)
        v, t, ms = qb.sap_tuning(16)
    finally:
        qb.set_sap_prec(32)
    assert rel_norm_err(psi, psi_ref) <= 1e-2
    assert rel_norm_err(rho, rho_ref) <= 3e-2
    assert t > 0 and ms > 0.0
    # the returned residual is the residual of the returned solution
    dpsi = qb.dirac_ref("Dw", 32, 0.01, psi)
    assert rel_norm_err(eta - dpsi, rho) <= 3e-2


def test_half_cycles_tiny_residual(setup):
    """A residual of 1e-12 (far below the FP16 range) gives the same
    relative result as a unit one: only the operator is stored in FP16."""
    eta = setup.source(32).astype(np.float32)
    qb.set_sap_prec(16)
    try:
        p1, r1 = qb.sap_ref(0.0, 1, 4, np.zeros_like(eta), eta)
        p2, r2 = qb.sap_ref(0.0, 1, 4, np.zeros_like(eta), (eta * np.float32(1e-12)).astype(np.float32))
    finally:
        qb.set_sap_prec(32)
    assert rel_norm_err(p2 * 1e12, p1) <= 1e-3
    assert rel_norm_err(r2 * 1e12, r1) <= 1e-3


def test_half_sap_gcr(setup):
    eta = setup.source(33)
    qb.set_sap_parms(setup.bs, 1, 4, 5)
    _, _, ifail32, st32 = qb.sap_gcr(16, 256, 0, 1e-10, 0.0, eta)
    qb.set_sap_prec(16)
    try:
        psi, rho, ifail, st = qb.sap_gcr(16, 256, 0, 1e-10, 0.0, eta)
    finally:
        qb.set_sap_prec(32)
        qb.set_sap_parms(setup.bs, 1, 4, 3)
    assert ifail == ifail32 == 0
    assert st <= st32 + max(1, st32 // 2), (st, st32)
    r = eta - setup.ref.dirac_dble(0, 0.0, psi)
    assert np.linalg.norm(r) / np.linalg.norm(eta) <= 1.5e-10
