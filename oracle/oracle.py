"""ctypes binding of the CPU restatement oracle (oracle/liboracle.so) and the
conversions between the reference's storage order and the oracle's
lexicographic one.  Test infrastructure only."""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            import importlib.util
            spec = importlib.util.spec_from_file_location("build_oracle", os.path.join(HERE, "build_oracle.py"))
            m = importlib.util.module_from_spec(spec)
            spec.loader.exec_module(m)
            m.build()
        L = C.CDLL(LIB)
        vp, i, d, f = C.c_void_p, C.c_int, C.c_double, C.c_float
        L.or_dirac_dble.argtypes = [vp, i, d, i, vp, vp, vp, vp, vp]
        L.or_dirac.argtypes = [vp, i, f, i, vp, vp, vp, vp, vp]
        L.or_inv_pauli.argtypes = [d, vp, vp]
        L.or_sw_term.argtypes = [vp, d, d, vp, vp]
        L.or_sap.argtypes = [vp, vp, f, i, i, i, vp, vp, vp, vp, vp]
        L.or_sap_gcr.argtypes = [vp, vp, i, i, i, i, d, vp, vp, vp, vp, i, i, i, d, d, vp, vp, vp, vp]
        L.or_sap_gcr.restype = d
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _L(L):
    return np.ascontiguousarray(L, dtype=np.int32)


# ---------------------------------------------------------- layout changes
def lex_index(L):
    return np.arange(L[0] * L[1] * L[2] * L[3])


def spinor_ref2lex(q, ipt):
    return np.ascontiguousarray(np.asarray(q).reshape(-1, 24)[ipt].reshape(-1))


def spinor_lex2ref(x, ipt):
    out = np.empty_like(np.asarray(x).reshape(-1, 24))
    out[ipt] = np.asarray(x).reshape(-1, 24)
    return out.reshape(-1)


def pauli_ref2lex(sw, ipt):
    return np.ascontiguousarray(np.asarray(sw).reshape(-1, 72)[ipt].reshape(-1))


def links_ref2lex(ud, ipt, L):
    """Forward links U(x,mu) per lexicographic site from the reference's
    8-links-per-odd-site array (main/README.global:229-262)."""
    V = len(ipt)
    ud = np.asarray(ud).reshape(-1, 18)
    out = np.empty((V, 4, 18))
    xs = np.array(np.unravel_index(np.arange(V), L)).T
    for mu in range(4):
        ix = ipt
        odd = ix >= V // 2
        xu = xs.copy()
        xu[:, mu] = (xu[:, mu] + 1) % L[mu]
        iy = ipt[np.ravel_multi_index(xu.T, L)]
        slot = np.where(odd, 8 * (ix - V // 2) + 2 * mu, 8 * (iy - V // 2) + 2 * mu + 1)
        out[:, mu] = ud[slot]
    return out.reshape(-1)


# ---------------------------------------------------------- restated ops
def dirac_dble(L, op, mu, tm_eo, U, sw, swi, s, r=None):
    s = np.ascontiguousarray(s, dtype=np.float64)
    r = np.zeros_like(s) if r is None else np.array(r, dtype=np.float64, copy=True)
    swi = sw if swi is None else swi
    lib().or_dirac_dble(_p(_L(L)), op, mu, tm_eo, _p(U), _p(sw), _p(swi), _p(s), _p(r))
    return r


def dirac(L, op, mu, tm_eo, U, sw, swi, s, r=None):
    s = np.ascontiguousarray(s, dtype=np.float32)
    r = np.zeros_like(s) if r is None else np.array(r, dtype=np.float32, copy=True)
    sw = np.ascontiguousarray(sw, dtype=np.float32)
    swi = sw if swi is None else np.ascontiguousarray(swi, dtype=np.float32)
    lib().or_dirac(_p(_L(L)), op, mu, tm_eo, _p(U), _p(sw), _p(swi), _p(s), _p(r))
    return r


def inv_pauli(mu, u):
    u = np.ascontiguousarray(u, dtype=np.float64)
    out = np.zeros(36)
    f = lib().or_inv_pauli(mu, _p(u), _p(out))
    return out, f


def invert_field(sw):
    sw = np.asarray(sw).reshape(-1, 36)
    out = np.empty_like(sw)
    fails = 0
    for i in range(sw.shape[0]):
        out[i], f = inv_pauli(0.0, sw[i])
        fails |= f
    return out.reshape(-1), fails


def sw_term(L, csw, m0, U):
    V = L[0] * L[1] * L[2] * L[3]
    sw = np.zeros(V * 72)
    lib().or_sw_term(_p(_L(L)), csw, m0, _p(np.ascontiguousarray(U)), _p(sw))
    return sw


def sap(L, bs, mu, isolv, nmr, tm_eo, U, sw32, swi32, psi, rho):
    psi = np.array(psi, dtype=np.float32, copy=True)
    rho = np.array(rho, dtype=np.float32, copy=True)
    lib().or_sap(_p(_L(L)), _p(_L(bs)), mu, isolv, nmr, tm_eo, _p(U), _p(sw32), _p(swi32), _p(psi), _p(rho))
    return psi, rho


def sap_gcr(L, bs, isolv, nmr, ncy, tm_eo, U, swd, sw32, swi32, nkv, nmx, istop, res, mu, eta):
    eta = np.ascontiguousarray(eta, dtype=np.float64)
    psi = np.zeros_like(eta)
    ifail = C.c_int(0)
    status = C.c_int(0)
    rho = lib().or_sap_gcr(_p(_L(L)), _p(_L(bs)), isolv, nmr, ncy, tm_eo, 0.0, _p(U), _p(swd), _p(sw32),
                           _p(swi32), nkv, nmx, istop, res, mu, _p(eta), _p(psi), C.byref(ifail), C.byref(status))
    return psi, rho, ifail.value, status.value
