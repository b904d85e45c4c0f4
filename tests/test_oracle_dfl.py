"""Pin the deflation conventions of the device code against the reference
(oracle/_ref): the order of the DFL blocks in a little vector, the layout of
a little vector (Ns complex numbers per block) and the orthonormality of the
block basis that dfl_modes/dfl_subspace produce.  CPU only.

The device code (openqcd-2.4.2_b200/csrc/dfl.cu) orders the blocks as the
reference's block grid does (modules/block/blk_grid.c): the blocks of colour
(sum of block coordinates) 0 first, then colour 1, each in lexicographic
order of the block coordinates with the last one running fastest."""
import numpy as np
import pytest

import reflib

L = (8, 8, 8, 8)
BS = (4, 4, 4, 4)
NS = 8

pytestmark = pytest.mark.skipif(not reflib.ensure_built(L), reason="reference oracle library not available")


def block_order(L, bs):
    nb = [L[m] // bs[m] for m in range(4)]
    coords = [(a, b, c, d) for a in range(nb[0]) for b in range(nb[1]) for c in range(nb[2]) for d in range(nb[3])]
    return [i for i, x in enumerate(coords) if sum(x) % 2 == 0] + [i for i, x in enumerate(coords) if sum(x) % 2]


@pytest.fixture(scope="module")
def ref():
    r = reflib.RefLib(L)
    r.init(bc=3, seed=1234, csw=1.5, m0=-0.2, eoflg=0)
    r.gen_links(0.4, 1234)
    assert r.sw_term(0) == 0
    r.set_sap_parms(BS, 1, 4, 5)
    r.dfl_init(BS, NS, kappa=1.0 / (2.0 * 3.8), ninv=5, nmr=4, ncy=4)
    f, _ = r.dfl_modes(7)
    assert f == 0
    return r


def block_sites(r):
    ipt = r.ipt()
    x = np.indices(L).reshape(4, -1).T
    lex = ((x[:, 0] * L[1] + x[:, 1]) * L[2] + x[:, 2]) * L[3] + x[:, 3]
    nb = [L[m] // BS[m] for m in range(4)]
    blk = (((x[:, 0] // BS[0]) * nb[1] + x[:, 1] // BS[1]) * nb[2] + x[:, 2] // BS[2]) * nb[3] + x[:, 3] // BS[3]
    return [ipt[lex[blk == b]] for b in block_order(L, BS)]


def test_block_order_and_s2vd(ref):
    sites = block_sites(ref)
    B = np.stack([ref.dfl_get_basis(l).reshape(ref.vol, 12, 2) for l in range(NS)])
    B = B[..., 0] + 1j * B[..., 1]
    s = np.random.default_rng(1).standard_normal((ref.vol, 24)).astype(np.float32)
    sc = s.reshape(ref.vol, 12, 2)
    sc = sc[..., 0] + 1j * sc[..., 1]
    vd = np.array([[np.vdot(B[l, ix].ravel(), sc[ix].ravel()) for l in range(NS)] for ix in sites])
    vd_ref = ref.dfl_s2vd(s.ravel()).view(np.complex128).reshape(len(sites), NS)
    assert np.abs(vd - vd_ref).max() <= 2e-6 * np.abs(vd_ref).max()


def test_basis_orthonormal(ref):
    sites = block_sites(ref)
    B = np.stack([ref.dfl_get_basis(l).reshape(ref.vol, 12, 2) for l in range(NS)]).astype(np.float64)
    B = B[..., 0] + 1j * B[..., 1]
    for ix in sites:
        G = np.einsum("lsc,ksc->lk", B[:, ix].conj(), B[:, ix])
        assert np.abs(G - np.eye(NS)).max() <= 1e-6


def test_vd2s_inverse_of_s2vd(ref):
    vd = np.random.default_rng(2).standard_normal(2 * ref.nv)
    back = ref.dfl_s2vd(ref.dfl_vd2s(vd))
    assert np.abs(back - vd).max() <= 1e-5 * np.abs(vd).max()
