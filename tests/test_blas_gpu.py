"""Drop-in BLAS-1 (salg.c, salg_dble.c) and the generic flexible GCR solver
(fgcr.c) against the reference.

Products: FP64 in double-double like the reference's qflt sums, compared to
1e-15 relative; FP32 products accumulate in double in both codes but the
reference rounds each 3-vector product to float first, so 1e-6.
"""
import ctypes as C

import numpy as np
import pytest

import openqcd_b200 as qb
from helpers import Setup

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    return Setup((8, 8, 8, 8), (4, 4, 4, 4), eps=0.4, csw=1.5, m0=0.0)


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def dd(q):
    return q.q[0] + q.q[1]


@pytest.mark.parametrize("where", ["host", "device"])
def test_spinor_prod_dble(setup, where):
    L = qb.lib()
    V = setup.vol
    s, r = setup.source(1), setup.source(2)
    ref = setup.ref.spinor_prod_dble(s, r)
    ref_n = setup.ref.norm_square_dble(s)
    if where == "host":
        ps, pr = _p(s), _p(r)
    else:
        ps = L.b200_dev_alloc(s.nbytes)
        pr = L.b200_dev_alloc(r.nbytes)
        qb.check(L.b200_memcpy(ps, _p(s), s.nbytes))
        qb.check(L.b200_memcpy(pr, _p(r), r.nbytes))
    z = L.spinor_prod_dble(V, 0, ps, pr)
    n = L.norm_square_dble(V, 0, ps)
    assert abs(dd(z.re) - (ref[0] + ref[1])) <= 1e-15 * abs(ref[0])
    assert abs(dd(z.im) - (ref[2] + ref[3])) <= 1e-15 * abs(ref[0])
    assert abs(dd(n) - (ref_n[0] + ref_n[1])) <= 1e-15 * ref_n[0]
    if where == "device":
        L.b200_dev_free(ps)
        L.b200_dev_free(pr)


def test_icom_threads(setup):
    """With icom & 2 the fields span vol sites per thread times NTHREAD."""
    L = qb.lib()
    s = setup.source(3)
    full = dd(L.norm_square_dble(setup.vol, 0, _p(s)))
    qb.check(L.b200_set_nthread(8))
    try:
        per = dd(L.norm_square_dble(setup.vol // 8, 3, _p(s)))
        part = dd(L.norm_square_dble(setup.vol // 8, 1, _p(s)))
    finally:
        L.b200_set_nthread(1)
    assert per == full
    assert part < full


def test_single_precision_products(setup):
    L = qb.lib()
    s, r = setup.source(4).astype(np.float32), setup.source(5).astype(np.float32)
    ref = setup.ref.spinor_prod(s, r)
    z = L.spinor_prod(setup.vol, 0, _p(s), _p(r))
    n = L.norm_square(setup.vol, 0, _p(s))
    assert abs(z.re - ref[0]) <= 1e-6 * abs(ref[0])
    assert abs(n - setup.ref.norm_square(s)) <= 1e-6 * n


def test_axpy_scale_normalize(setup):
    L = qb.lib()
    s, r = setup.source(6), setup.source(7)
    x = s.copy()
    L.mulc_spinor_add_dble(setup.vol, 0, _p(x), _p(r), qb.ComplexD(0.3, -0.7))
    zz = (0.3 - 0.7j)
    want = (s.view(np.complex128) + zz * r.view(np.complex128)).view(np.float64)
    assert np.allclose(x, want, rtol=0, atol=1e-14)
    L.scale_dble(setup.vol, 0, 2.5, _p(x))
    assert np.allclose(x, 2.5 * want, rtol=0, atol=1e-13)
    nrm = L.normalize_dble(setup.vol, 0, _p(x))
    assert abs(nrm - np.linalg.norm(2.5 * want)) <= 1e-12 * nrm
    assert abs(np.linalg.norm(x) - 1.0) <= 1e-14


def test_generic_fgcr_with_sap_preconditioner(setup):
    """fgcr(vol, Dop, Mop, ...) with Dop = Dw_dble and Mop = ncy SAP cycles on
    host arrays, all through the library's drop-in calls: the sap_gcr
    recursion rebuilt by the caller (sap_gcr.c:120-133)."""
    L = qb.lib()
    V = setup.vol
    mu, nkv = 0.0, 16
    qb.set_sap_parms((4, 4, 4, 4), 1, 4, 5)

    def dop(s, r):
        L.Dw_dble(mu, s, r)

    def mop(k, rho, phi, chi):
        nb = V * 24 * 4
        C.memset(phi, 0, nb)
        C.memmove(chi, rho, nb)
        for _ in range(5):
            L.sap(mu, 1, 4, phi, chi)
        rh = np.ctypeslib.as_array((C.c_float * (V * 24)).from_address(rho))
        ch = np.ctypeslib.as_array((C.c_float * (V * 24)).from_address(chi))
        ch[:] = rh - ch

    Dop = qb.DOP_T(dop)
    Mop = qb.MOP_T(mop)
    ws = [np.zeros(V * 24, dtype=np.float32) for _ in range(2 * nkv + 1)]
    wsd = [np.zeros(V * 24)]
    wsp = (C.c_void_p * len(ws))(*[w.ctypes.data for w in ws])
    wsdp = (C.c_void_p * 1)(wsd[0].ctypes.data)
    eta = setup.source(8)
    psi = np.zeros_like(eta)
    status = C.c_int(0)
    rn = L.fgcr(V, Dop, Mop, wsp, wsdp, nkv, 256, 0, 1e-10, _p(eta), _p(psi), C.byref(status))
    _, _, ifail, st = qb.sap_gcr(nkv, 256, 0, 1e-10, mu, eta)
    res = np.linalg.norm(eta - setup.ref.dirac_dble(0, mu, psi)) / np.linalg.norm(eta)
    assert status.value > 0 and abs(status.value - st) <= 1
    assert rn <= 1e-10 * np.linalg.norm(eta) * 1.00001
    assert res <= 1.5e-10
