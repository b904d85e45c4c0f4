"""ctypes binding of the reference CPU oracle (oracle/_ref/<tag>/libref.so).

Test infrastructure: imported only by tests/, the smoke check and the CPU
baseline of bench.py.  One library per lattice geometry; a process can load
several (each has its own copy of the reference's module state).
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

# lattice -> thread-local lattice (the reference's Lx_TRD), NTHREAD = V / V_TRD
GEOMETRIES = {
    (8, 8, 8, 8): (4, 4, 4, 8),          # 8 threads
    (8, 8, 8, 16): (4, 4, 4, 8),         # 16 threads
    (16, 8, 8, 8): (4, 4, 4, 8),         # 16 threads
    (16, 16, 16, 16): (8, 8, 8, 8),      # 16 threads
    (12, 12, 12, 12): (6, 6, 12, 12),    # 4 threads (6^4 blocks)
    (64, 32, 32, 32): (32, 16, 16, 32),  # 8 threads
}


def tag(L, T, portable=False):
    vol = L[0] * L[1] * L[2] * L[3]
    return "%dx%dx%dx%d_t%d%s" % (L[0], L[1], L[2], L[3], vol // (T[0] * T[1] * T[2] * T[3]),
                                 "_c" if portable else "")


def lib_path(L, T=None, portable=False):
    T = T or GEOMETRIES[tuple(L)]
    return os.path.join(HERE, "_ref", tag(L, T, portable), "libref.so")


def available(L, T=None, portable=False):
    return os.path.exists(lib_path(L, T, portable))


def ensure_built(L, T=None, ref="/root/reference", portable=False):
    """Build the library for this geometry if it is missing and the reference
    sources are present (they are not on the GPU machines).  portable=True
    selects the reference's plain-C code paths (no AVX inline assembly)."""
    T = T or GEOMETRIES[tuple(L)]
    p = lib_path(L, T, portable)
    if not os.path.exists(p) and os.path.isdir(ref):
        import importlib.util
        spec = importlib.util.spec_from_file_location("build_ref", os.path.join(HERE, "build_ref.py"))
        m = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(m)
        m.build(list(L), list(T), ref, verbose=False, portable=portable)
    return os.path.exists(p)


class RefLib:
    def __init__(self, L, T=None, portable=False, private=False):
        """private: load a private copy of the library (its own parameter
        data base, e.g. for a second SW type in the same process; the
        reference's set_lat_parms can be called only once per instance)."""
        T = T or GEOMETRIES[tuple(L)]
        self.L = tuple(L)
        self.portable = portable
        path = lib_path(L, T, portable)
        if not os.path.exists(path):
            raise RuntimeError("reference oracle not built: " + path)
        if private:
            import shutil
            import tempfile
            d = tempfile.mkdtemp(prefix="refcopy")
            cp = os.path.join(d, os.path.basename(path))
            shutil.copyfile(path, cp)
            path = cp
        self.lib = C.CDLL(path)
        l = self.lib
        l.ref_init.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_int]
        l.ref_set_sw_parms.argtypes = [C.c_double]
        l.ref_set_tm_parms.argtypes = [C.c_int]
        l.ref_set_sap_parms.argtypes = [C.c_int] * 7
        l.ref_gen_links.argtypes = [C.c_double, C.c_int]
        l.ref_random_ud.argtypes = [C.c_int]
        l.ref_sw_term.argtypes = [C.c_int]
        l.ref_random_sd.argtypes = [C.c_int, C.c_double, C.c_void_p]
        l.ref_dirac_dble.argtypes = [C.c_int, C.c_double, C.c_void_p, C.c_void_p]
        l.ref_dirac.argtypes = [C.c_int, C.c_float, C.c_void_p, C.c_void_p]
        l.ref_sap.argtypes = [C.c_float, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
        l.ref_sap_gcr.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_void_p, C.c_void_p,
                                  C.c_void_p, C.c_void_p]
        l.ref_sap_gcr.restype = C.c_double
        l.ref_time_dirac.argtypes = [C.c_int, C.c_double, C.c_int]
        l.ref_time_dirac.restype = C.c_double
        self.vol = l.ref_volume()
        self.nthread = l.ref_nthread()

    @staticmethod
    def _p(a):
        return a.ctypes.data_as(C.c_void_p)

    def init(self, bc=3, seed=1234, csw=1.5, m0=0.0, eoflg=0, isw=0, theta=None):
        """theta: the spatial phase angles of set_bc_parms (taken by the
        first init of a library instance only)"""
        if theta is not None:
            self.lib.ref_set_theta.argtypes = [C.c_double] * 3
            self.lib.ref_set_theta(*[float(t) for t in theta])
        self.lib.ref_init_isw.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int]
        self.lib.ref_init_isw(bc, seed, csw, m0, eoflg, isw)

    def set_sw_parms(self, m0):
        self.lib.ref_set_sw_parms(m0)

    def set_tm_parms(self, eoflg):
        self.lib.ref_set_tm_parms(eoflg)

    def set_sap_parms(self, bs, isolv, nmr, ncy):
        self.lib.ref_set_sap_parms(bs[0], bs[1], bs[2], bs[3], isolv, nmr, ncy)

    def gen_links(self, eps, seed):
        self.lib.ref_gen_links(eps, seed)

    def sw_term(self, which=0):
        return self.lib.ref_sw_term(which)

    def ipt(self):
        out = np.zeros(self.vol, dtype=np.int32)
        self.lib.ref_get_ipt(self._p(out))
        return out

    def ud(self):
        out = np.zeros(4 * self.vol * 18)
        self.lib.ref_get_ud(self._p(out))
        return out

    def set_ud(self, ud):
        ud = np.ascontiguousarray(ud, dtype=np.float64)
        self.lib.ref_set_ud(self._p(ud))

    def swd(self):
        out = np.zeros(2 * self.vol * 36)
        self.lib.ref_get_swd(self._p(out))
        return out

    def random_sd(self, seed, sigma=1.0):
        out = np.zeros(self.vol * 24)
        self.lib.ref_random_sd(seed, sigma, self._p(out))
        return out

    def dirac_dble(self, op, mu, s, r=None):
        s = np.ascontiguousarray(s, dtype=np.float64)
        r = np.zeros_like(s) if r is None else np.array(r, dtype=np.float64, copy=True)
        self.lib.ref_dirac_dble(op, mu, self._p(s), self._p(r))
        return r

    def dirac(self, op, mu, s, r=None):
        s = np.ascontiguousarray(s, dtype=np.float32)
        r = np.zeros_like(s) if r is None else np.array(r, dtype=np.float32, copy=True)
        self.lib.ref_dirac(op, mu, self._p(s), self._p(r))
        return r

    def sap(self, mu, isolv, nmr, ncy, psi, rho):
        psi = np.array(psi, dtype=np.float32, copy=True)
        rho = np.array(rho, dtype=np.float32, copy=True)
        f = self.lib.ref_sap(mu, isolv, nmr, ncy, self._p(psi), self._p(rho))
        return psi, rho, f

    def sap_gcr(self, nkv, nmx, istop, res, mu, eta):
        eta = np.ascontiguousarray(eta, dtype=np.float64)
        psi = np.zeros_like(eta)
        ifail = C.c_int(0)
        status = C.c_int(0)
        rho = self.lib.ref_sap_gcr(nkv, nmx, istop, res, mu, self._p(eta), self._p(psi), C.byref(ifail),
                                   C.byref(status))
        return psi, rho, ifail.value, status.value

    def time_dirac(self, op, mu, n):
        return self.lib.ref_time_dirac(op, mu, n)

    def time_dirac_src(self, mu, s, n):
        """seconds for n applications of Dw_dble to s; returns (seconds, Dw_dble s)"""
        s = np.ascontiguousarray(s, dtype=np.float64)
        r = np.zeros_like(s)
        f = self.lib.ref_time_dirac_src
        f.argtypes = [C.c_double, C.c_void_p, C.c_void_p, C.c_int]
        f.restype = C.c_double
        t = f(mu, self._p(s), self._p(r), n)
        return t, r

    def apply_sw_dble(self, vol, mu, m, s):
        m = np.ascontiguousarray(m, dtype=np.float64)
        s = np.ascontiguousarray(s, dtype=np.float64)
        r = np.zeros_like(s)
        self.lib.ref_apply_sw_dble.argtypes = [C.c_int, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p]
        self.lib.ref_apply_sw_dble(vol, mu, self._p(m), self._p(s), self._p(r))
        return r

    def apply_sw(self, vol, mu, m, s):
        m = np.ascontiguousarray(m, dtype=np.float32)
        s = np.ascontiguousarray(s, dtype=np.float32)
        r = np.zeros_like(s)
        self.lib.ref_apply_sw.argtypes = [C.c_int, C.c_float, C.c_void_p, C.c_void_p, C.c_void_p]
        self.lib.ref_apply_sw(vol, mu, self._p(m), self._p(s), self._p(r))
        return r

    def apply_swinv_dble(self, vol, mu, m, s):
        m = np.ascontiguousarray(m, dtype=np.float64)
        s = np.ascontiguousarray(s, dtype=np.float64)
        r = np.zeros_like(s)
        self.lib.ref_apply_swinv_dble.argtypes = [C.c_int, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p]
        f = self.lib.ref_apply_swinv_dble(vol, mu, self._p(m), self._p(s), self._p(r))
        return r, f

    def inv_pauli_dble(self, mu, m):
        m = np.ascontiguousarray(m, dtype=np.float64)
        im = np.zeros(36)
        self.lib.ref_inv_pauli_dble.argtypes = [C.c_double, C.c_void_p, C.c_void_p]
        f = self.lib.ref_inv_pauli_dble(mu, self._p(m), self._p(im))
        return im, f

    def spinor_prod_dble(self, s, r):
        s = np.ascontiguousarray(s, dtype=np.float64)
        r = np.ascontiguousarray(r, dtype=np.float64)
        out = np.zeros(4)
        self.lib.ref_spinor_prod_dble.argtypes = [C.c_void_p] * 3
        self.lib.ref_spinor_prod_dble(self._p(s), self._p(r), self._p(out))
        return out

    def norm_square_dble(self, s):
        s = np.ascontiguousarray(s, dtype=np.float64)
        out = np.zeros(2)
        self.lib.ref_norm_square_dble.argtypes = [C.c_void_p] * 2
        self.lib.ref_norm_square_dble(self._p(s), self._p(out))
        return out

    def spinor_prod(self, s, r):
        s = np.ascontiguousarray(s, dtype=np.float32)
        r = np.ascontiguousarray(r, dtype=np.float32)
        out = np.zeros(2, dtype=np.float32)
        self.lib.ref_spinor_prod.argtypes = [C.c_void_p] * 3
        self.lib.ref_spinor_prod(self._p(s), self._p(r), self._p(out))
        return out

    def norm_square(self, s):
        s = np.ascontiguousarray(s, dtype=np.float32)
        self.lib.ref_norm_square.argtypes = [C.c_void_p]
        self.lib.ref_norm_square.restype = C.c_float
        return self.lib.ref_norm_square(self._p(s))

    # ------------------------------------------------------------ deflation
    def dfl_init(self, bs, Ns, nkv=16, nmx=256, res=1e-2, nmx_gcr=24, res_gcr=1e-2, kappa=0.125, mu=0.0,
                 ninv=5, nmr=4, ncy=4):
        l = self.lib
        l.ref_dfl_init.argtypes = [C.c_int] * 7 + [C.c_double, C.c_int, C.c_double, C.c_double, C.c_double,
                                                    C.c_int, C.c_int, C.c_int]
        self.nv = l.ref_dfl_init(bs[0], bs[1], bs[2], bs[3], Ns, nkv, nmx, res, nmx_gcr, res_gcr, kappa, mu,
                                 ninv, nmr, ncy)
        self.Ns = Ns
        return self.nv

    def dfl_modes(self, seed):
        status = (C.c_int * 2)()
        self.lib.ref_dfl_modes.argtypes = [C.c_int, C.c_void_p]
        f = self.lib.ref_dfl_modes(seed, status)
        return f, list(status)

    def dfl_random_fields(self, seed, Ns):
        """the start fields of dfl_modes after start_ranlux(0, seed), [Ns, V*24] FP32"""
        out = np.zeros((Ns, self.vol * 24), dtype=np.float32)
        self.lib.ref_dfl_random_fields.argtypes = [C.c_int, C.c_int, C.c_void_p]
        self.lib.ref_dfl_random_fields(seed, Ns, self._p(out))
        return out

    def dfl_subspace(self, modes):
        m = np.ascontiguousarray(np.concatenate([np.asarray(x, dtype=np.float32) for x in modes]))
        self.lib.ref_dfl_subspace.argtypes = [C.c_int, C.c_void_p]
        self.lib.ref_dfl_subspace(len(modes), self._p(m))

    def dfl_get_basis(self, l):
        out = np.zeros(self.vol * 24, dtype=np.float32)
        self.lib.ref_dfl_get_basis.argtypes = [C.c_int, C.c_void_p]
        self.lib.ref_dfl_get_basis(l, self._p(out))
        return out

    def dfl_s2vd(self, s):
        s = np.ascontiguousarray(s, dtype=np.float32)
        vd = np.zeros(2 * self.nv)
        self.lib.ref_dfl_s2vd.argtypes = [C.c_void_p, C.c_void_p]
        self.lib.ref_dfl_s2vd(self._p(s), self._p(vd))
        return vd

    def dfl_vd2s(self, vd):
        vd = np.ascontiguousarray(vd, dtype=np.float64)
        s = np.zeros(self.vol * 24, dtype=np.float32)
        self.lib.ref_dfl_vd2s.argtypes = [C.c_void_p, C.c_void_p]
        self.lib.ref_dfl_vd2s(self._p(vd), self._p(s))
        return s

    def little(self, which, mu, v, w=None):
        v = np.ascontiguousarray(v, dtype=np.float64)
        w = np.zeros_like(v) if w is None else np.array(w, dtype=np.float64, copy=True)
        self.lib.ref_little.argtypes = [C.c_int, C.c_double, C.c_void_p, C.c_void_p]
        f = self.lib.ref_little(which, mu, self._p(v), self._p(w))
        return w, f

    def little32(self, which, mu, v, w=None):
        v = np.ascontiguousarray(v, dtype=np.float32)
        w = np.zeros_like(v) if w is None else np.array(w, dtype=np.float32, copy=True)
        self.lib.ref_little32.argtypes = [C.c_int, C.c_double, C.c_void_p, C.c_void_p]
        self.lib.ref_little32(which, mu, self._p(v), self._p(w))
        return w

    def dfl_get_lmode(self, l, nv):
        out = np.zeros(2 * nv, dtype=np.float32)
        self.lib.ref_dfl_get_lmode.argtypes = [C.c_int, C.c_void_p]
        self.lib.ref_dfl_get_lmode(l, self._p(out))
        return out

    def ltl_modes(self, mu, ns):
        m = np.zeros(2 * ns * ns)
        self.lib.ref_ltl_modes.argtypes = [C.c_double, C.c_void_p]
        f = self.lib.ref_ltl_modes(mu, self._p(m))
        return m, f

    def dfl_proj(self, which, v, w=None):
        v = np.array(v, dtype=np.float64, copy=True)
        w = np.zeros_like(v) if w is None else np.array(w, dtype=np.float64, copy=True)
        self.lib.ref_dfl_proj.argtypes = [C.c_int, C.c_void_p, C.c_void_p]
        self.lib.ref_dfl_proj(which, self._p(v), self._p(w))
        return v, w

    def dfl_Lv(self, v):
        v = np.array(v, dtype=np.float32, copy=True)
        self.lib.ref_dfl_Lv.argtypes = [C.c_void_p]
        self.lib.ref_dfl_Lv(self._p(v))
        return v

    def ltl_gcr(self, mu, eta):
        eta = np.ascontiguousarray(eta, dtype=np.float64)
        psi = np.zeros_like(eta)
        ifail = C.c_int(0)
        status = (C.c_int * 2)()
        self.lib.ref_ltl_gcr.argtypes = [C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        self.lib.ref_ltl_gcr.restype = C.c_double
        rho = self.lib.ref_ltl_gcr(mu, self._p(eta), self._p(psi), C.byref(ifail), status)
        return psi, rho, ifail.value, list(status)

    def dfl_sap_gcr(self, nkv, nmx, istop, res, mu, eta):
        eta = np.ascontiguousarray(eta, dtype=np.float64)
        psi = np.zeros_like(eta)
        ifail = C.c_int(0)
        status = (C.c_int * 3)()
        self.lib.ref_dfl_sap_gcr.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_void_p,
                                             C.c_void_p, C.c_void_p, C.c_void_p]
        self.lib.ref_dfl_sap_gcr.restype = C.c_double
        rho = self.lib.ref_dfl_sap_gcr(nkv, nmx, istop, res, mu, self._p(eta), self._p(psi), C.byref(ifail),
                                       status)
        return psi, rho, ifail.value, list(status)

    def time_dfl_sap_gcr(self, nkv, nmx, res, mu, eta):
        eta = np.ascontiguousarray(eta, dtype=np.float64)
        status = (C.c_int * 3)()
        self.lib.ref_time_dfl_sap_gcr.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_void_p,
                                                  C.c_void_p]
        self.lib.ref_time_dfl_sap_gcr.restype = C.c_double
        t = self.lib.ref_time_dfl_sap_gcr(nkv, nmx, res, mu, self._p(eta), status)
        return t, list(status)

    def time_sap_gcr(self, nkv, nmx, res, mu, eta):
        eta = np.ascontiguousarray(eta, dtype=np.float64)
        status = (C.c_int * 3)()
        self.lib.ref_time_sap_gcr.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_void_p, C.c_void_p]
        self.lib.ref_time_sap_gcr.restype = C.c_double
        t = self.lib.ref_time_sap_gcr(nkv, nmx, res, mu, self._p(eta), status)
        return t, list(status)

    # ------------------------------------------------------------- archives
    def export_cnfg(self, path):
        self.lib.ref_export_cnfg.argtypes = [C.c_char_p]
        self.lib.ref_export_cnfg(path.encode())

    def import_cnfg(self, path):
        self.lib.ref_import_cnfg.argtypes = [C.c_char_p]
        self.lib.ref_import_cnfg(path.encode())

    def export_sfld(self, path, eo, sd):
        sd = np.ascontiguousarray(sd, dtype=np.float64)
        self.lib.ref_export_sfld.argtypes = [C.c_char_p, C.c_int, C.c_void_p]
        self.lib.ref_export_sfld(path.encode(), eo, self._p(sd))

    def import_sfld(self, path, eo):
        out = np.zeros(self.vol * 24)
        self.lib.ref_import_sfld.argtypes = [C.c_char_p, C.c_int, C.c_void_p]
        self.lib.ref_import_sfld(path.encode(), eo, self._p(out))
        return out

    def plaq_sum(self):
        self.lib.ref_plaq_sum.restype = C.c_double
        return self.lib.ref_plaq_sum()

    def tmcg(self, nmx, istop, res, mu, eta, eo=False, psi0=None):
        eta = np.ascontiguousarray(eta, dtype=np.float64)
        psi = np.zeros_like(eta) if psi0 is None else np.array(psi0, dtype=np.float64, copy=True)
        ifail = C.c_int(0)
        status = C.c_int(0)
        self.lib.ref_tmcg.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p]
        self.lib.ref_tmcg.restype = C.c_double
        rho = self.lib.ref_tmcg(1 if eo else 0, nmx, istop, res, mu, self._p(eta), self._p(psi), C.byref(ifail),
                                C.byref(status))
        return psi, rho, ifail.value, status.value

    def tmcgm(self, nmx, istop, res, mu, eta, psi0=None):
        """tmcgm for len(mu) <= 64 shifts; returns (solutions, ifail, status)"""
        eta = np.ascontiguousarray(eta, dtype=np.float64)
        mu = np.ascontiguousarray(mu, dtype=np.float64)
        res = np.ascontiguousarray(res, dtype=np.float64)
        nmu = len(mu)
        assert nmu <= 64
        psi = np.zeros((nmu, eta.size)) if psi0 is None else np.array(psi0, dtype=np.float64, copy=True)
        ifail = C.c_int(0)
        status = C.c_int(0)
        self.lib.ref_tmcgm.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_void_p, C.c_void_p]
        self.lib.ref_tmcgm.restype = None
        self.lib.ref_tmcgm(nmx, istop, self._p(res), nmu, self._p(mu), self._p(eta), self._p(psi), C.byref(ifail),
                           C.byref(status))
        return [psi[k] for k in range(nmu)], ifail.value, status.value
