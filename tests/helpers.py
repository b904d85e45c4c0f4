"""Shared set-up for the parity tests: reference fields from the CPU oracle,
loaded into the device library through its C interface."""
import numpy as np

import openqcd_b200 as qb
import reflib

OPS = ["Dw", "Dwee", "Dwoo", "Dwoe", "Dweo", "Dwhat"]


def site_rel_err(a, b, vol):
    """max over sites of |a(x)-b(x)| / |b(x)| (24 reals per site)."""
    a = np.asarray(a, dtype=np.float64).reshape(vol, 24)
    b = np.asarray(b, dtype=np.float64).reshape(vol, 24)
    d = np.linalg.norm(a - b, axis=1)
    n = np.linalg.norm(b, axis=1)
    mask = n > 0
    if not mask.any():
        return float(d.max())
    return float((d[mask] / n[mask]).max()) if mask.all() else max(float((d[mask] / n[mask]).max()), float(d[~mask].max()))


def rel_norm_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


class Setup:
    """Reference fields on lattice L (links exp(eps X), SW term), and the
    device library loaded with the same fields."""

    def __init__(self, L, bs=(4, 4, 4, 4), eps=0.4, csw=1.5, m0=0.0, seed=1234, eoflg=0, portable=False, isw=0,
                 theta=None, private=False):
        assert reflib.ensure_built(L, portable=portable), "reference oracle library missing for %s" % (L,)
        # the exponential SW type and phase angles need their own instance
        # of the reference (set_lat_parms and set_bc_parms are called once
        # per instance)
        self.ref = reflib.RefLib(L, portable=portable, private=private or isw != 0 or theta is not None)
        self.ref.init(bc=3, seed=seed, csw=csw, m0=m0, eoflg=eoflg, isw=isw, theta=theta)
        self.ref.gen_links(eps, seed)
        assert self.ref.sw_term(0) == 0
        self.L = tuple(L)
        self.bs = tuple(bs)
        self.vol = self.ref.vol
        self.ipt = self.ref.ipt()
        self.ud = self.ref.ud()
        self.swd = self.ref.swd()
        qb.geometry(L, bs, self.ipt)
        qb.set_parms(csw, m0, eoflg, isw=isw)
        qb.set_bc_theta(theta if theta is not None else (0.0, 0.0, 0.0))
        qb.upload_ud(self.ud)
        self.sw_fail = qb.upload_swd(self.swd)

    def source(self, seed):
        return self.ref.random_sd(seed)
