"""Pin the CPU restatement (oracle/qcd_oracle.c) against the reference itself
(oracle/_ref, the reference's own modules compiled here) on identical fields.
CPU only; these are the oracle's credentials."""
import numpy as np
import pytest

import oracle as orc
import reflib
from helpers import OPS, site_rel_err

L = (8, 8, 8, 8)
BS = (4, 4, 4, 4)

pytestmark = pytest.mark.skipif(not reflib.ensure_built(L), reason="reference oracle library not available")


@pytest.fixture(scope="module")
def f():
    r = reflib.RefLib(L)
    r.init(bc=3, seed=1234, csw=1.5, m0=-0.05, eoflg=0)
    r.gen_links(0.4, 1234)
    assert r.sw_term(0) == 0
    ipt = r.ipt()
    d = dict(ref=r, ipt=ipt, vol=r.vol)
    d["U"] = orc.links_ref2lex(r.ud(), ipt, L)
    d["swd_ref"] = r.swd()
    d["sw"] = orc.pauli_ref2lex(d["swd_ref"], ipt)
    d["swi"], fails = orc.invert_field(d["sw"])
    assert fails == 0
    return d


def test_sw_term(f):
    sw = orc.sw_term(L, 1.5, -0.05, f["U"])
    a, b = sw.reshape(-1, 36), f["sw"].reshape(-1, 36)
    assert (np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)).max() <= 1e-14


def test_inverse(f):
    r = f["ref"]
    r.sw_term(3)
    inv_ref = orc.pauli_ref2lex(r.swd(), f["ipt"])
    r.sw_term(0)
    a, b = f["swi"].reshape(-1, 36), inv_ref.reshape(-1, 36)
    assert (np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)).max() <= 1e-12


@pytest.mark.parametrize("op", OPS)
@pytest.mark.parametrize("mu", [0.0, 0.137])
def test_dirac_dble(f, op, mu):
    r, ipt, vol = f["ref"], f["ipt"], f["vol"]
    s = r.random_sd(11)
    r0 = r.random_sd(12)
    k = OPS.index(op)
    if op == "Dwhat":
        r.sw_term(2)
    out_ref = r.dirac_dble(k, mu, s, r0)
    if op == "Dwhat":
        r.sw_term(0)
    out = orc.dirac_dble(L, k, mu, 0, f["U"], f["sw"], f["swi"], orc.spinor_ref2lex(s, ipt),
                         orc.spinor_ref2lex(r0, ipt))
    assert site_rel_err(orc.spinor_lex2ref(out, ipt), out_ref, vol) <= 1e-13


@pytest.mark.parametrize("op", OPS)
def test_dirac_single(f, op):
    r, ipt, vol = f["ref"], f["ipt"], f["vol"]
    s = r.random_sd(21).astype(np.float32)
    r0 = r.random_sd(22).astype(np.float32)
    k = OPS.index(op)
    if op == "Dwhat":
        r.sw_term(2)
    out_ref = r.dirac(k, 0.137, s, r0)
    if op == "Dwhat":
        r.sw_term(0)
    out = orc.dirac(L, k, 0.137, 0, f["U"], f["sw"], f["swi"], orc.spinor_ref2lex(s, ipt), orc.spinor_ref2lex(r0, ipt))
    assert site_rel_err(orc.spinor_lex2ref(out, ipt), out_ref, vol) <= 2e-6


@pytest.fixture(scope="module")
def fc(f):
    """The reference built from its plain-C code paths (no AVX assembly)."""
    if not reflib.ensure_built(L, portable=True):
        pytest.skip("portable reference oracle not available")
    r = reflib.RefLib(L, portable=True)
    r.init(bc=3, seed=1234, csw=1.5, m0=-0.05, eoflg=0)
    r.gen_links(0.4, 1234)
    r.set_ud(f["ref"].ud())      # bit-identical links for both builds
    assert r.sw_term(0) == 0
    return r


@pytest.mark.parametrize("isolv", [1, 0])
@pytest.mark.parametrize("nmr", [1, 4])
def test_sap_cycle(f, fc, isolv, nmr):
    """Against the reference's plain-C build: FP32 rounding only."""
    r, ipt = fc, f["ipt"]
    eta = r.random_sd(3).astype(np.float32)
    r.set_sap_parms(BS, isolv, nmr, 2)
    psi_ref, rho_ref, _ = r.sap(0.05, isolv, nmr, 2, np.zeros_like(eta), eta)
    psi = np.zeros(eta.size, dtype=np.float32)
    rho = orc.spinor_ref2lex(eta, ipt)
    for _ in range(2):
        psi, rho = orc.sap(L, BS, 0.05, isolv, nmr, 0, f["U"], f["sw"].astype(np.float32),
                           f["swi"].astype(np.float32), psi, rho)
    for a, b in ((psi, psi_ref), (rho, rho_ref)):
        a = orc.spinor_lex2ref(a, ipt)
        assert np.linalg.norm(a - b) / np.linalg.norm(b) <= 2e-6


@pytest.mark.parametrize("isolv", [1, 0])
def test_sap_cycle_avx_build(f, isolv):
    """Against the AVX build, whose MR step length uses the approximate
    reciprocal vrcpss (modules/sap/blk_solv.c:291-300, relative error up to
    1.5 * 2^-12): agreement to that level only."""
    r, ipt = f["ref"], f["ipt"]
    eta = r.random_sd(3).astype(np.float32)
    r.set_sap_parms(BS, isolv, 4, 2)
    psi_ref, rho_ref, _ = r.sap(0.05, isolv, 4, 2, np.zeros_like(eta), eta)
    psi = np.zeros(eta.size, dtype=np.float32)
    rho = orc.spinor_ref2lex(eta, ipt)
    for _ in range(2):
        psi, rho = orc.sap(L, BS, 0.05, isolv, 4, 0, f["U"], f["sw"].astype(np.float32),
                           f["swi"].astype(np.float32), psi, rho)
    for a, b in ((psi, psi_ref), (rho, rho_ref)):
        a = orc.spinor_lex2ref(a, ipt)
        assert np.linalg.norm(a - b) / np.linalg.norm(b) <= 2e-3


def test_sap_gcr(f):
    r, ipt = f["ref"], f["ipt"]
    eta = r.random_sd(7)
    r.set_sap_parms(BS, 1, 4, 5)
    psi_ref, rho_ref, ifail_ref, st_ref = r.sap_gcr(16, 256, 0, 1e-10, 0.0, eta)
    psi, rho, ifail, st = orc.sap_gcr(L, BS, 1, 4, 5, 0, f["U"], f["sw"], f["sw"].astype(np.float32),
                                      f["swi"].astype(np.float32), 16, 256, 0, 1e-10, 0.0,
                                      orc.spinor_ref2lex(eta, ipt))
    psi = orc.spinor_lex2ref(psi, ipt)
    assert ifail == ifail_ref == 0
    assert abs(st - st_ref) <= 1
    res = eta - r.dirac_dble(0, 0.0, psi)
    assert np.linalg.norm(res) / np.linalg.norm(eta) <= 1.5e-10
    assert np.linalg.norm(psi - psi_ref) / np.linalg.norm(psi_ref) <= 1e-8
