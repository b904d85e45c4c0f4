"""The batched restriction and prolongation (b200_dfl_s2vd_multi /
b200_dfl_vd2s_multi) against the reference's dfl_s2vd and dfl_vd2s
(modules/dfl/dfl_subspace.c:83, :126), field by field, on the same block
basis (the reference's dfl_subspace of random modes, uploaded to the
device).  Four fields per pass run on the tensor cores (mma.sync with TF32
head/tail operands) or on the CUDA cores, one or two on the CUDA cores; all
must meet the bar of
the single-field routines: 2e-6 relative to the largest component (the
reference computes in FP32 and rounds its inner products to FP32).  Ns = 8,
20, 28 and 40 cover one, two (with padded rows) and three row tiles of 16
basis vectors, and one to ten k-steps of the prolongation.

The batched Awhat_dble (the little operator of the batched little solver:
four vectors per pass on the tensor cores with the hop matrices rounded to
FP32) against the reference's Awhat_dble (modules/little/Aw_dble.c:361):
1e-6 relative in norm (FP32 matrices; the reference's own FP32 little
operators are held to 1e-5), and the FP64 passes of the same call to
1e-12."""
import numpy as np
import pytest

import openqcd_b200 as qb
from helpers import Setup, rel_norm_err

pytestmark = pytest.mark.gpu

L = (8, 8, 8, 8)
BS = (4, 4, 4, 4)
M0 = -0.2
KAPPA = 1.0 / (2.0 * (4.0 + M0))


@pytest.fixture(scope="module", params=[8, 20, 28, 40])
def st(request):
    Ns = request.param
    # set_dfl_parms may be called once per instance of the reference
    s = Setup(L, BS, eps=0.4, csw=1.5, m0=M0, private=True)
    s.ref.set_sap_parms(BS, 1, 4, 5)
    s.nv = s.ref.dfl_init(BS, Ns, nkv=16, nmx=256, res=1e-2, nmx_gcr=24, res_gcr=1e-2, kappa=KAPPA, mu=0.0,
                          ninv=5, nmr=4, ncy=4)
    rng = np.random.default_rng(100 + Ns)
    s.ref.dfl_subspace([rng.standard_normal(s.vol * 24).astype(np.float32) for _ in range(Ns)])
    qb.set_sap_parms(BS, 1, 4, 5)
    assert qb.set_dfl_parms(BS, Ns) == s.nv
    for l in range(Ns):
        qb.dfl_set_basis(l, s.ref.dfl_get_basis(l))
    s.Ns = Ns
    return s


KINDS = [(4, True), (4, False), (2, False), (1, False)]   # fields per pass, tensor cores


@pytest.mark.parametrize("tile,tc", KINDS)
@pytest.mark.parametrize("nr", [4, 5, 8])
def test_s2vd_multi(st, nr, tile, tc):
    qb.set_rhs_tiles(tile, tile, tc, tc)
    rng = np.random.default_rng(7 * nr + tile)
    fields = [rng.standard_normal(st.vol * 24).astype(np.float32) for _ in range(nr)]
    vds = qb.dfl_s2vd_multi(fields, st.nv)
    worst = 0.0
    for f, vd in zip(fields, vds):
        ref = st.ref.dfl_s2vd(f)
        worst = max(worst, np.abs(vd - ref).max() / np.abs(ref).max())
    print("Ns %d nr %d tile %d tc %d: max error %.2e" % (st.Ns, nr, tile, tc, worst))
    assert worst <= 2e-6, worst


@pytest.mark.parametrize("tile,tc", KINDS)
@pytest.mark.parametrize("nr", [4, 6])
def test_vd2s_multi(st, nr, tile, tc):
    qb.set_rhs_tiles(tile, tile, tc, tc)
    rng = np.random.default_rng(11 * nr + tile)
    vds = [rng.standard_normal(2 * st.nv) for _ in range(nr)]
    fs = qb.dfl_vd2s_multi(vds, st.vol)
    worst = 0.0
    for vd, f in zip(vds, fs):
        ref = st.ref.dfl_vd2s(vd)
        worst = max(worst, np.abs(f - ref).max() / np.abs(ref).max())
    print("Ns %d nr %d tile %d tc %d: max error %.2e" % (st.Ns, nr, tile, tc, worst))
    assert worst <= 2e-6, worst


def test_tiles_back_to_autotuner(st):
    qb.set_rhs_tiles(0, 0)
    t = qb.rhs_tiles()
    assert t["restrict"] == 0 and t["prolong"] == 0
    rng = np.random.default_rng(3)
    fields = [rng.standard_normal(st.vol * 24).astype(np.float32) for _ in range(4)]
    vds = qb.dfl_s2vd_multi(fields, st.nv)
    assert qb.rhs_tiles()["restrict"] in (1, 2, 4)
    ref = st.ref.dfl_s2vd(fields[2])
    assert np.abs(vds[2] - ref).max() <= 2e-6 * np.abs(ref).max()


@pytest.mark.parametrize("nr", [4, 5])
def test_awhat_multi(st, nr):
    rng = np.random.default_rng(31 + nr)
    vs = [rng.standard_normal(2 * st.nv) for _ in range(nr)]
    w0 = [rng.standard_normal(2 * st.nv) for _ in range(nr)]
    mu = 0.01
    qb.little(1, mu, vs[0])                 # set_Awhat(mu) on the device
    ws = qb.Awhat_multi(vs, w0)
    for r in range(nr):
        ref, f = st.ref.little(1, mu, vs[r], w0[r])
        assert f == 0
        err = rel_norm_err(ws[r], ref)
        print("Ns %d nr %d vector %d: relative error %.2e" % (st.Ns, nr, r, err))
        assert err <= (1e-6 if r < 4 else 1e-12), (r, err)



@pytest.fixture(scope="module")
def st6():
    """6^4 blocks on 12^4, Ns = 28: 648 sites per block parity (81 groups of 8
    sites over the warps of the tensor-core kernels, 486 prolongation tiles)"""
    L6, BS6, Ns = (12, 12, 12, 12), (6, 6, 6, 6), 28
    s = Setup(L6, BS6, eps=0.4, csw=1.5, m0=M0, portable=True, private=True)
    s.ref.set_sap_parms(BS6, 1, 4, 5)
    s.nv = s.ref.dfl_init(BS6, Ns, nkv=16, nmx=256, res=1e-2, nmx_gcr=24, res_gcr=1e-2, kappa=KAPPA, mu=0.0,
                          ninv=5, nmr=4, ncy=4)
    rng = np.random.default_rng(606)
    s.ref.dfl_subspace([rng.standard_normal(s.vol * 24).astype(np.float32) for _ in range(Ns)])
    qb.set_sap_parms(BS6, 1, 4, 5)
    assert qb.set_dfl_parms(BS6, Ns) == s.nv
    for l in range(Ns):
        qb.dfl_set_basis(l, s.ref.dfl_get_basis(l))
    s.Ns = Ns
    return s


@pytest.mark.parametrize("tile,tc", [(4, True), (4, False)])
def test_multi_6x6x6x6_blocks(st6, tile, tc):
    qb.set_rhs_tiles(tile, tile, tc, tc)
    rng = np.random.default_rng(61 + tile + tc)
    fields = [rng.standard_normal(st6.vol * 24).astype(np.float32) for _ in range(4)]
    vds = qb.dfl_s2vd_multi(fields, st6.nv)
    for f, vd in zip(fields, vds):
        ref = st6.ref.dfl_s2vd(f)
        assert np.abs(vd - ref).max() <= 2e-6 * np.abs(ref).max()
    vin = [rng.standard_normal(2 * st6.nv) for _ in range(4)]
    fs = qb.dfl_vd2s_multi(vin, st6.vol)
    for vd, f in zip(vin, fs):
        ref = st6.ref.dfl_vd2s(vd)
        assert np.abs(f - ref).max() <= 2e-6 * np.abs(ref).max()
    qb.little(1, 0.01, vin[0])
    ws = qb.Awhat_multi(vin)
    for v, w in zip(vin, ws):
        ref, f = st6.ref.little(1, 0.01, v)
        assert f == 0 and rel_norm_err(w, ref) <= 1e-6
