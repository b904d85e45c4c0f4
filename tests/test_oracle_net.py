"""Pin the CPU oracle of the learned preconditioner's network
(oracle/ptnet.py): its gradient against central finite differences, its
layer adjoint against the inner-product identity, and gauge equivariance of
the network (M[U^om] om psi = om M[U] psi for a random gauge transformation
om).  CPU only, small random lattice."""
import numpy as np

import ptnet

L = (4, 4, 2, 4)


def setup(seed=0):
    rng = np.random.default_rng(seed)
    U = ptnet.random_links(L, rng)
    nb = ptnet.neighbours(L)
    n = sum(2 * 9 * ptnet.CH[l] * ptnet.CH[l + 1] for l in range(3))
    w = 0.3 * rng.standard_normal(n)
    V = int(np.prod(L))
    r = rng.standard_normal((V, 4, 3)) + 1j * rng.standard_normal((V, 4, 3))
    e = rng.standard_normal((V, 4, 3)) + 1j * rng.standard_normal((V, 4, 3))
    return rng, U, nb, w, r, e


def test_gradient_finite_differences():
    rng, U, nb, w, r, e = setup(1)
    loss, g = ptnet.loss_grad(U, nb, ptnet.unpack(w), r, e)
    idx = rng.choice(len(w), 40, replace=False)
    h = 1e-6
    for k in idx:
        wp, wm = w.copy(), w.copy()
        wp[k] += h
        wm[k] -= h
        lp, _ = ptnet.loss_grad(U, nb, ptnet.unpack(wp), r, e)
        lm, _ = ptnet.loss_grad(U, nb, ptnet.unpack(wm), r, e)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(fd)), (k, fd, g[k])


def test_layer_adjoint():
    rng, U, nb, w, r, e = setup(2)
    W = ptnet.unpack(w)[1]
    V = int(np.prod(L))
    x = rng.standard_normal((V, 8, 3)) + 1j * rng.standard_normal((V, 8, 3))
    y = rng.standard_normal((V, 8, 3)) + 1j * rng.standard_normal((V, 8, 3))
    lhs = np.vdot(y, ptnet.layer(U, nb, W, x))
    rhs = np.vdot(ptnet.layer_adjoint(U, nb, W, y), x)
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs)


def test_gauge_equivariance():
    rng, U, nb, w, r, e = setup(3)
    Ws = ptnet.unpack(w)
    V = int(np.prod(L))
    om = ptnet.random_links(L, rng)[:, 0]
    y = ptnet.forward(U, nb, Ws, r)[-1]
    Ug = ptnet.gauge_transform(U, nb, om)
    yg = ptnet.forward(Ug, nb, Ws, np.einsum("xab,xib->xia", om, r))[-1]
    assert np.abs(yg - np.einsum("xab,xib->xia", om, y)).max() <= 1e-12 * np.abs(y).max()
