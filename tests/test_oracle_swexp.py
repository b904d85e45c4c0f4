"""The reference's exponential SW term, pinned: a private instance of the
reference library run with isw = 1 next to one with isw = 0 on the same
gauge field gives c expm(A) with A = (SW_0 - c)/c traceless Hermitian
(sw_term.c:46-49), checked with scipy's matrix exponential."""
import numpy as np
import pytest
import scipy.linalg

import reflib

L = (8, 8, 8, 8)
CSW, M0 = 1.7, -0.1


def unpack(u):
    A = np.zeros((6, 6), dtype=complex)
    A[np.diag_indices(6)] = u[:6]
    k = 6
    for i in range(6):
        for j in range(i + 1, 6):
            A[i, j] = u[k] + 1j * u[k + 1]
            A[j, i] = np.conj(A[i, j])
            k += 2
    return A


@pytest.fixture(scope="module")
def refs():
    if not reflib.ensure_built(L):
        pytest.skip("reference oracle library missing")
    r0 = reflib.RefLib(L, private=True)
    r0.init(bc=3, seed=77, csw=CSW, m0=M0, isw=0)
    r0.gen_links(0.4, 77)
    r1 = reflib.RefLib(L, private=True)
    r1.init(bc=3, seed=77, csw=CSW, m0=M0, isw=1)
    r1.gen_links(0.4, 77)
    r0.sw_term(0)
    r1.sw_term(0)
    return r0, r1


def test_reference_swexp_is_matrix_exponential(refs):
    r0, r1 = refs
    assert np.array_equal(r0.ud(), r1.ud())
    s0 = r0.swd().reshape(-1, 36)
    s1 = r1.swd().reshape(-1, 36)
    c = 4.0 + M0
    rng = np.random.default_rng(5)
    for n in rng.choice(len(s0), 64, replace=False):
        A = (unpack(s0[n]) - c * np.eye(6)) / c
        assert abs(np.trace(A)) < 1e-13
        B = c * scipy.linalg.expm(A)
        assert np.linalg.norm(unpack(s1[n]) - B) <= 1e-13 * np.linalg.norm(B)
