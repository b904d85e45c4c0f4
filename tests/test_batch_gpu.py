"""Several right-hand sides solved together (b200_dev_gcr_batch, no reference
counterpart).  Every system runs the reference's algorithm (fgcr with SAP,
modules/sap/sap_gcr.c:140, or with deflated SAP, modules/dfl/dfl_sap_gcr.c:353)
on its own Krylov space, so each must reach the FP64 true residual 1e-10,
checked with the reference's Dw_dble, in the number of steps of the
single-system solver give or take one, with a solution equal to the
single-system one to 1e-8 (the batched solver orthogonalises by classical
Gram-Schmidt in fused passes, and its restriction and little solver sum in
another order).  Systems of different twisted masses and a zero source
share a batch (with deflation, one little operator per mass); systems
leave it as they converge."""
import numpy as np
import pytest

import openqcd_b200 as qb
from helpers import Setup, rel_norm_err

pytestmark = pytest.mark.gpu

L = (8, 8, 8, 8)
BS = (4, 4, 4, 4)
NS = 8
M0 = -0.2


@pytest.fixture(scope="module")
def setup():
    s = Setup(L, BS, eps=0.4, csw=1.5, m0=M0)
    qb.set_sap_parms(BS, 1, 4, 5)
    return s


def dev(prec, arr=None):
    f = qb.DevField(prec)
    if arr is not None:
        f.from_ref(arr)
    return f


def true_res(setup, mu, psi, eta):
    r = eta - setup.ref.dirac_dble(0, mu, psi)
    return np.linalg.norm(r) / np.linalg.norm(eta)


def test_plain_batch_matches_single(setup):
    mus = [0.0, 0.02, 0.08]
    etas = [setup.source(41 + i) for i in range(3)]
    singles = []
    for mu, eta in zip(mus, etas):
        e, p = dev(64, eta), dev(64)
        rho, ifail, st = qb.dev_sap_gcr(16, 256, 0, 1e-10, mu, e, p)
        singles.append((p.to_ref(setup.vol), st))
    E = [dev(64, e) for e in etas]
    P = [dev(64) for _ in etas]
    rho, ifail, st, _ = qb.dev_gcr_batch(16, 256, 0, 1e-10, mus, E, P)
    assert ifail == [0, 0, 0]
    for i in range(3):
        psi = P[i].to_ref(setup.vol)
        assert abs(st[i] - singles[i][1]) <= 1, (st, [x[1] for x in singles])
        assert rel_norm_err(psi, singles[i][0]) <= 1e-8
        assert true_res(setup, mus[i], psi, etas[i]) <= 1.5e-10


def test_plain_batch_zero_source(setup):
    eta = setup.source(45)
    E = [dev(64, np.zeros_like(eta)), dev(64, eta)]
    P = [dev(64, eta), dev(64)]
    rho, ifail, st, _ = qb.dev_gcr_batch(16, 256, 0, 1e-10, [0.0, 0.0], E, P)
    assert rho[0] == 0.0 and ifail == [0, 0]
    assert not P[0].to_ref(setup.vol).any()
    assert true_res(setup, 0.0, P[1].to_ref(setup.vol), eta) <= 1.5e-10


@pytest.fixture(scope="module")
def dfl(setup):
    setup.ref.set_sap_parms(BS, 1, 4, 5)
    setup.nv = setup.ref.dfl_init(BS, NS, nkv=16, nmx=256, res=1e-2, nmx_gcr=24, res_gcr=1e-2,
                                  kappa=1.0 / (2.0 * (4.0 + M0)), mu=0.0, ninv=5, nmr=4, ncy=4)
    f, _ = setup.ref.dfl_modes(7)
    assert f == 0
    assert qb.set_dfl_parms(BS, NS) == setup.nv
    qb.set_dfl_pro_parms(16, 256, 1e-2, 24, 1e-2)
    for l in range(NS):
        qb.dfl_set_basis(l, setup.ref.dfl_get_basis(l))
    return setup


@pytest.mark.parametrize("nr", [1, 5])
def test_dfl_batch_matches_single(dfl, nr):
    mu = 0.01
    etas = [dfl.source(51 + i) for i in range(nr)]
    singles = []
    for eta in etas:
        e, p = dev(64, eta), dev(64)
        rho, ifail, st = qb.dev_dfl_sap_gcr(16, 256, 0, 1e-10, mu, e, p)
        assert ifail == 0
        singles.append((p.to_ref(dfl.vol), st[0]))
    E = [dev(64, e) for e in etas]
    P = [dev(64) for _ in etas]
    rho, ifail, st, lst = qb.dev_gcr_batch(16, 256, 0, 1e-10, [mu] * nr, E, P, dfl=True)
    assert ifail == [0] * nr
    for i in range(nr):
        psi = P[i].to_ref(dfl.vol)
        assert abs(st[i] - singles[i][1]) <= 1, (st, [x[1] for x in singles])
        assert lst[i] > 0
        assert rel_norm_err(psi, singles[i][0]) <= 1e-8
        assert true_res(dfl, mu, psi, etas[i]) <= 1.5e-10


def test_dfl_batch_mixed_masses(dfl):
    """systems of different twisted masses share one deflated batch: each
    mass gets its own little operator, the restriction, prolongation and
    SAP are shared; every system equals its single-system solve"""
    mus = [0.0, 0.01, 0.0, 0.03]
    etas = [dfl.source(60 + i) for i in range(len(mus))]
    singles = []
    for mu, eta in zip(mus, etas):
        e, p = dev(64, eta), dev(64)
        rho, ifail, st = qb.dev_dfl_sap_gcr(16, 256, 0, 1e-10, mu, e, p)
        assert ifail == 0
        singles.append((p.to_ref(dfl.vol), st[0]))
    E = [dev(64, e) for e in etas]
    P = [dev(64) for _ in etas]
    rho, ifail, st, lst = qb.dev_gcr_batch(16, 256, 0, 1e-10, mus, E, P, dfl=True)
    assert ifail == [0] * len(mus)
    for i, mu in enumerate(mus):
        psi = P[i].to_ref(dfl.vol)
        assert abs(st[i] - singles[i][1]) <= 1, (st, [x[1] for x in singles])
        assert rel_norm_err(psi, singles[i][0]) <= 1e-8
        assert true_res(dfl, mu, psi, etas[i]) <= 1.5e-10
    qb.release_workspace()


def test_point_source(setup):
    f = dev(64)
    x = (3, 1, 4, 2)
    f.point(x, 2, 1)
    q = f.to_ref(setup.vol).reshape(setup.vol, 24)
    lex = ((x[0] * L[1] + x[1]) * L[2] + x[2]) * L[3] + x[3]
    ix = setup.ipt[lex]
    assert q[ix, 2 * (3 * 2 + 1)] == 1.0 and np.count_nonzero(q) == 1
    g = qb.DevField(32)
    g.point(x, 3, 2)
    q = g.to_ref(setup.vol).reshape(setup.vol, 24)
    assert q[ix, 2 * (3 * 3 + 2)] == 1.0 and np.count_nonzero(q) == 1


@pytest.mark.parametrize("n", [1, 3, 6])
def test_dirac_multi(setup, n):
    """Dw on several FP32 fields at once equals Dw on each (FP32, 2e-6 per
    site), and the fused r = sub - Dw s equals the difference."""
    from helpers import site_rel_err
    mu = 0.03
    S = [dev(32, setup.source(70 + i).astype(np.float32)) for i in range(n)]
    U = [dev(32, setup.source(80 + i).astype(np.float32)) for i in range(n)]
    R = [qb.DevField(32) for _ in range(n)]
    Q = [qb.DevField(32) for _ in range(n)]
    qb.dev_dirac_multi(mu, S, R)
    qb.dev_dirac_multi(mu, S, Q, U)
    for i in range(n):
        one = qb.DevField(32)
        qb.dev_dirac("Dw", mu, S[i], one)
        ref = one.to_ref(setup.vol)
        assert site_rel_err(R[i].to_ref(setup.vol), ref, setup.vol) <= 2e-6
        diff = U[i].to_ref(setup.vol).astype(np.float64) - ref
        assert site_rel_err(Q[i].to_ref(setup.vol), diff, setup.vol) <= 2e-6


def test_rhs_tile_autotuner(setup):
    """After a deflated batched solve the RHS-tile autotuner has timed the
    restriction and prolongation with 1, 2 and 4 fields per pass on the CUDA
    cores and 4 on the tensor cores, and kept the fastest."""
    t = qb.rhs_tiles()
    assert t["restrict"] in (1, 2, 4) and t["prolong"] in (1, 2, 4), t
    assert all(m > 0 for m in t["restrict_ms"] + t["prolong_ms"]), t
    for k in ("restrict", "prolong"):
        kind = {1: 0, 2: 1, 4: 3 if t[k + "_tc"] else 2}[t[k]]
        assert t[k + "_ms"][kind] == min(t[k + "_ms"]), t
