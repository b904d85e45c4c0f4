"""The learned preconditioner (csrc/net.cu, no reference counterpart)
against its CPU oracle (oracle/ptnet.py, itself pinned by finite
differences and gauge equivariance on the CPU), on the reference's gauge
field: forward pass to 1e-5 (FP32 arithmetic), FP16-rounded weights within
3e-3 of FP32 ones, loss to 1e-5 and gradient to 1e-4 (relative norms).
Training on the device must lower the loss, and the trained network,
as the flexible-GCR preconditioner, must reach the FP64 residual 1e-10
(checked with the reference's Dw_dble) in fewer steps than GCR without a
preconditioner; with SAP added after it, in no more steps than SAP alone
plus two."""
import numpy as np
import pytest

import openqcd_b200 as qb
import oracle as orc
import ptnet
from helpers import Setup

pytestmark = pytest.mark.gpu

L = (8, 8, 8, 8)
BS = (4, 4, 4, 4)


@pytest.fixture(scope="module")
def setup():
    s = Setup(L, BS, eps=0.4, csw=1.5, m0=-0.2)
    qb.set_sap_parms(BS, 1, 4, 5)
    s.U = ptnet.links_from_lex(orc.links_ref2lex(s.ud, s.ipt, L))
    s.nb = ptnet.neighbours(L)
    yield s
    qb.set_precond(0)


def to_dev(s, ch):
    f = qb.DevField(32)
    f.from_ref(orc.spinor_lex2ref(ptnet.channels_to_spinor_lex(ch), s.ipt).astype(np.float32))
    return f


def from_dev(s, f):
    return ptnet.spinor_lex_to_channels(orc.spinor_ref2lex(f.to_ref(s.vol), s.ipt))


def rand_ch(s, seed):
    rng = np.random.default_rng(seed)
    c = rng.standard_normal((s.vol, 4, 3)) + 1j * rng.standard_normal((s.vol, 4, 3))
    return c.astype(np.complex64).astype(np.complex128)


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_forward(setup):
    qb.net_init(5, 0.25)
    w = qb.net_get_weights()
    r = rand_ch(setup, 1)
    rd, yd = to_dev(setup, r), qb.DevField(32)
    qb.net_apply(rd, yd, half=False)
    y = ptnet.forward(setup.U, setup.nb, ptnet.unpack(w), r)[-1]
    assert rel(from_dev(setup, yd), y) <= 1e-5
    y16 = qb.DevField(32)
    qb.net_apply(rd, y16, half=True)
    assert rel(from_dev(setup, y16), y) <= 3e-3


def test_gradient(setup):
    rng = np.random.default_rng(7)
    w = (0.2 * rng.standard_normal(qb.net_nweights())).astype(np.float32)
    qb.net_set_weights(w)
    r, e = rand_ch(setup, 2), rand_ch(setup, 3)
    loss, g = qb.net_grad(to_dev(setup, r), to_dev(setup, e))
    loss_o, g_o = ptnet.loss_grad(setup.U, setup.nb, ptnet.unpack(w), r, e)
    assert abs(loss - loss_o) <= 1e-5 * loss_o
    assert rel(g, g_o) <= 1e-4


def iterations(setup, kind, eta):
    qb.set_precond(kind)
    psi, rho, ifail, st = qb.sap_gcr(16, 2048, 0, 1e-10, 0.0, eta)
    qb.set_precond(0)
    r = eta - setup.ref.dirac_dble(0, 0.0, psi)
    assert ifail == 0
    assert np.linalg.norm(r) / np.linalg.norm(eta) <= 1.5e-10
    return st


def test_train_and_precondition(setup):
    n = 48
    rs = [qb.DevField(32) for _ in range(n)]
    es = [qb.DevField(32) for _ in range(n)]
    qb.set_precond(0)
    qb.net_make_pairs(rs, es, 0.0, 1e-6, seed=11)
    qb.net_init(3, 0.25)
    hist = qb.net_train(rs, es, 300, 4, 3e-3, seed=5)
    assert np.isfinite(hist).all()
    assert hist[-30:].mean() < 0.6 * hist[:5].mean(), (hist[:5], hist[-30:])
    eta = setup.source(77)
    it_none = iterations(setup, 3, eta)
    it_net = iterations(setup, 1, eta)
    it_sap = iterations(setup, 0, eta)
    it_both = iterations(setup, 2, eta)
    print("GCR steps: none %d, network %d, SAP %d, network+SAP %d; loss %.3g -> %.3g"
          % (it_none, it_net, it_sap, it_both, hist[:5].mean(), hist[-30:].mean()))
    assert it_net < it_none
    assert it_both <= it_sap + 2


def test_sap_error_pairs_and_sap_plus_network(setup):
    """(residual, SAP-error) pairs: e + M_sap r solves D x = r (to the
    solver's residual); a network trained on them, added to SAP (kind 4),
    reaches the FP64 residual in no more steps than SAP alone plus two"""
    n = 32
    rs = [qb.DevField(32) for _ in range(n)]
    es = [qb.DevField(32) for _ in range(n)]
    qb.set_precond(0)
    qb.net_make_sap_pairs(rs, es, 0.0, 1e-6, seed=13)
    # check one pair: D (e + M_sap r) = r
    r = rs[0].to_ref(setup.vol).astype(np.float64)
    e = es[0].to_ref(setup.vol).astype(np.float64)
    psi, rho = qb.sap_ref(0.0, 1, 4, np.zeros_like(r, dtype=np.float32), r.astype(np.float32))
    for _ in range(4):   # ncy = 5 cycles in all, as the pairs were made
        psi, rho = qb.sap_ref(0.0, 1, 4, psi, rho)
    x = e + psi.astype(np.float64)
    res = np.linalg.norm(setup.ref.dirac_dble(0, 0.0, x) - r) / np.linalg.norm(r)
    assert res < 1e-4, res
    qb.net_init(5, 0.1)
    hist = qb.net_train(rs, es, 200, 4, 3e-3, seed=6)
    assert np.isfinite(hist).all()
    eta = setup.source(79)
    it_sap = iterations(setup, 0, eta)
    it_4 = iterations(setup, 4, eta)
    assert it_4 <= it_sap + 2, (it_4, it_sap)


def test_poisoned_network_falls_back_to_sap(setup):
    """a network with garbage weights: the network preconditioner (kind 1)
    and SAP plus network (kind 4) stall, drop the network after one step
    that reduces the residual by less than 10 %, and still reach the FP64
    residual 1e-10 through SAP"""
    w = qb.net_get_weights()
    rng = np.random.default_rng(3)
    try:
        qb.net_set_weights((50.0 * rng.standard_normal(w.size)).astype(np.float32))
        eta = setup.source(81)
        it_sap = iterations(setup, 0, eta)
        for kind in (1, 4):
            it = iterations(setup, kind, eta)     # asserts the true residual
            assert it <= 4 * it_sap + 8, (kind, it, it_sap)
    finally:
        qb.net_set_weights(w)
        qb.set_precond(0)
