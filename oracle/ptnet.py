"""CPU oracle (numpy, double precision) of the gauge-equivariant
parallel-transport network of the learned preconditioner
(openqcd-2.4.2_b200/csrc/net.cu).  Test infrastructure only: it checks the
device forward pass and the device gradients, and its own gradient is
checked against finite differences.

Fields are lexicographic (x3 fastest) arrays of shape (V, C, 3) complex:
C channels of colour triplets per site; a spinor field is C = 4 (its spin
components).  Links U have shape (V, 4, 3, 3), U[x, mu] the forward link.
A layer maps Cin to Cout channels:

    y_o(x) = sum_{d=0..8} sum_i W[d, o, i] (T_d psi_i)(x)
    T_0 psi(x) = psi(x)
    T_{1+2mu} psi(x) = U(x, mu) psi(x + mu)
    T_{2+2mu} psi(x) = U(x - mu, mu)^dag psi(x - mu)

The network is three layers, 4 -> 8 -> 8 -> 4 channels.
"""
import numpy as np

CH = (4, 8, 8, 4)


def neighbours(L):
    V = int(np.prod(L))
    x = np.array(np.unravel_index(np.arange(V), L)).T
    fwd, bwd = [], []
    for mu in range(4):
        y = x.copy()
        y[:, mu] = (y[:, mu] + 1) % L[mu]
        fwd.append(np.ravel_multi_index(y.T, L))
        y = x.copy()
        y[:, mu] = (y[:, mu] - 1) % L[mu]
        bwd.append(np.ravel_multi_index(y.T, L))
    return fwd, bwd


def links_from_lex(u_lex):
    """(V*4*18,) reals (the layout of oracle.links_ref2lex) -> (V, 4, 3, 3)."""
    a = np.asarray(u_lex, dtype=np.float64).reshape(-1, 4, 9, 2)
    return (a[..., 0] + 1j * a[..., 1]).reshape(-1, 4, 3, 3)


def transport(U, nb, d, psi):
    fwd, bwd = nb
    if d == 0:
        return psi
    mu = (d - 1) // 2
    if d % 2 == 1:
        return np.einsum("xab,xib->xia", U[:, mu], psi[fwd[mu]])
    y = bwd[mu]
    return np.einsum("xba,xib->xia", U[y, mu].conj(), psi[y])


def layer(U, nb, W, psi):
    return sum(np.einsum("oi,xic->xoc", W[d], transport(U, nb, d, psi)) for d in range(9))


def layer_adjoint(U, nb, W, g):
    """psi -> layer is linear; this is its adjoint, written out directly:
    (T_{+mu}^dag g)(y) = U(y-mu, mu)^dag g(y-mu), (T_{-mu}^dag g)(y) =
    U(y, mu) g(y+mu)."""
    fwd, bwd = nb
    out = np.einsum("oi,xoc->xic", W[0].conj(), g)
    for mu in range(4):
        h = np.einsum("oi,xoc->xic", W[1 + 2 * mu].conj(), g)
        y = bwd[mu]
        out = out + np.einsum("xba,xib->xia", U[y, mu].conj(), h[y])
        h = np.einsum("oi,xoc->xic", W[2 + 2 * mu].conj(), g)
        out = out + np.einsum("xab,xib->xia", U[:, mu], h[fwd[mu]])
    return out


def unpack(w):
    """packed float weights -> list of (9, Cout, Cin) complex arrays"""
    w = np.asarray(w, dtype=np.float64)
    out, k = [], 0
    for l in range(3):
        n = 9 * CH[l + 1] * CH[l]
        a = w[k:k + 2 * n].reshape(9, CH[l + 1], CH[l], 2)
        out.append(a[..., 0] + 1j * a[..., 1])
        k += 2 * n
    return out


def pack(Ws):
    return np.concatenate([np.stack([W.real, W.imag], axis=-1).reshape(-1) for W in Ws])


def forward(U, nb, Ws, psi):
    a = psi
    acts = [a]
    for W in Ws:
        a = layer(U, nb, W, a)
        acts.append(a)
    return acts


def loss_grad(U, nb, Ws, r, e):
    """loss |M r - e|^2/|e|^2 and its gradient w.r.t. Re W + i Im W,
    packed like the weights."""
    acts = forward(U, nb, Ws, r)
    res = acts[-1] - e
    e2 = np.vdot(e, e).real
    loss = np.vdot(res, res).real / e2
    g = 2.0 * res / e2
    grads = [None] * 3
    for l in (2, 1, 0):
        a = acts[l]
        grads[l] = np.stack([np.einsum("xoc,xic->oi", g, transport(U, nb, d, a).conj()) for d in range(9)])
        if l > 0:
            g = layer_adjoint(U, nb, Ws[l], g)
    return loss, pack(grads)


def spinor_lex_to_channels(x):
    """(V*24,) reals of a lexicographic spinor field -> (V, 4, 3) complex"""
    a = np.asarray(x, dtype=np.float64).reshape(-1, 4, 3, 2)
    return a[..., 0] + 1j * a[..., 1]


def channels_to_spinor_lex(c):
    return np.stack([c.real, c.imag], axis=-1).reshape(-1)


def random_links(L, rng):
    """Random SU(3)-like unitary links (QR of Gaussian matrices) for tests
    that need no reference field."""
    V = int(np.prod(L))
    z = rng.standard_normal((V, 4, 3, 3)) + 1j * rng.standard_normal((V, 4, 3, 3))
    q, r = np.linalg.qr(z)
    ph = np.diagonal(r, axis1=-2, axis2=-1)
    return q * (ph / np.abs(ph))[..., None, :]


def gauge_transform(U, nb, om):
    """U'(x, mu) = om(x) U(x, mu) om(x+mu)^dag"""
    fwd, _ = nb
    out = np.empty_like(U)
    for mu in range(4):
        out[:, mu] = om @ U[:, mu] @ om[fwd[mu]].conj().transpose(0, 2, 1)
    return out
