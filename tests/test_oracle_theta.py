"""The reference with phase angles theta (set_bc_parms, lat_parms.c:516):
a private instance of the reference library started with theta, on the same
seed as one without, holds the links of the other times exp(i theta[k-1]/N[k])
in direction k (set_ud_phase, modules/uflds/uflds.c:249-355), and the same
time links.  Pins the oracle hook the phase-angle device tests use."""
import numpy as np
import pytest

import reflib

L = (8, 8, 8, 8)
THETA = (0.5, -0.8, 1.3)


@pytest.fixture(scope="module")
def refs():
    if not reflib.ensure_built(L):
        pytest.skip("reference oracle library missing")
    out = []
    for th in (None, THETA):
        r = reflib.RefLib(L, private=True)
        r.init(bc=3, seed=1234, csw=1.5, m0=-0.1, theta=th)
        r.gen_links(0.4, 77)
        out.append(r.ud().reshape(-1, 8, 9, 2))
    return out


def test_theta_phase(refs):
    u0, u1 = (a[..., 0] + 1j * a[..., 1] for a in refs)
    assert np.array_equal(u0[:, :2], u1[:, :2])          # time links untouched
    for k in range(3):
        ph = np.exp(1j * THETA[k] / L[k + 1])
        assert np.abs(u1[:, 2 + 2 * k: 4 + 2 * k] - ph * u0[:, 2 + 2 * k: 4 + 2 * k]).max() < 1e-15
