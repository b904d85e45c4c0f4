"""Helpers of the domain-decomposition tests: the reference's storage order
of a global field cut into the x0-slabs of the ranks, and the rank process
that runs the library on its slab (the exchange of faces goes through the
host and gloo, so no kernel waits on another process).

Storage order (main/README.global): ipt[lex] = storage index, lex with x3
fastest and x0 slowest; ud holds U(x, mu) at slot 8 (ix - V/2) + 2 mu of the
odd site x and U(x - mu, mu) at slot 8 (ix - V/2) + 2 mu + 1; swd holds the
two Pauli matrices of site ix at 2 ix, 2 ix + 1; spinors are 24 reals per
site in storage order.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def coords(L):
    return np.indices(L).reshape(4, -1)


def ud_to_lex(ud, L, ipt):
    """forward links U(x, mu) [V, 4, 18] (lexicographic x) of a storage-order field"""
    V = int(np.prod(L))
    u = ud.reshape(4 * V, 18)
    x = coords(L)
    odd = (x.sum(axis=0) & 1) == 1
    out = np.empty((V, 4, 18))
    for mu in range(4):
        lx = np.nonzero(odd)[0]
        out[lx, mu] = u[8 * (ipt[lx] - V // 2) + 2 * mu]
        ev = np.nonzero(~odd)[0]
        y = x[:, ev].copy()
        y[mu] = (y[mu] + 1) % L[mu]
        ly = np.ravel_multi_index(tuple(y), L)
        out[ev, mu] = u[8 * (ipt[ly] - V // 2) + 2 * mu + 1]
    return out


def slab_ud(U, L, nproc, rank, ipt_loc):
    """storage-order gauge field of rank `rank`'s slab (local lattice
    L0/nproc x L1 x L2 x L3, storage order ipt_loc) of the global forward
    links U [V, 4, 18]: the backward links of the first plane's odd sites
    come from the slab below, as openQCD's local fields hold them"""
    L0 = L[0] // nproc
    Ll = (L0,) + tuple(L[1:])
    Vl = int(np.prod(Ll))
    x = coords(Ll)
    odd = np.nonzero(x.sum(axis=0) & 1)[0]
    xg = x[:, odd].copy()
    xg[0] += rank * L0
    base = 8 * (ipt_loc[odd].astype(np.int64) - Vl // 2)
    out = np.empty((4 * Vl, 18))
    for mu in range(4):
        out[base + 2 * mu] = U[np.ravel_multi_index(tuple(xg), L), mu]
        y = xg.copy()
        y[mu] = (y[mu] - 1) % L[mu]
        out[base + 2 * mu + 1] = U[np.ravel_multi_index(tuple(y), L), mu]
    return out.reshape(-1)


def slab_sites(flex, L, nproc, rank, ipt_loc):
    """storage-order site field (per-site rows of flex [V, k], lexicographic)
    of rank `rank`'s slab"""
    L0 = L[0] // nproc
    F = int(np.prod(L[1:]))
    part = flex[rank * L0 * F:(rank + 1) * L0 * F]
    out = np.empty_like(part)
    out[ipt_loc] = part
    return out


def even_first_ipt(L):
    x = coords(L)
    par = x.sum(axis=0) & 1
    order = np.argsort(par, kind="stable")
    ipt = np.empty(order.size, dtype=np.int32)
    ipt[order] = np.arange(order.size, dtype=np.int32)
    return ipt


def rank_main(rank, world, port, inp, outp):
    """One rank: its slab of the global fields from inp (an .npz), the
    library's operators and solvers under domain decomposition, results
    (storage order of the slab) to outp."""
    sys.path.insert(0, os.path.join(ROOT, "openqcd-2.4.2_b200"))
    import datetime

    import torch.distributed as dist

    import openqcd_b200 as qb
    d = dict(np.load(inp % rank))
    # a short timeout: a rank that fails ends the others' next exchange with an error
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    res = {}
    try:
        dd = qb.DomainDecomposition(transport="host")
        dd.install()
        Ll = tuple(int(v) for v in d["L_loc"])
        bs = tuple(int(v) for v in d["bs"])
        qb.geometry(Ll, bs, d["ipt"])
        qb.set_parms(float(d["csw"]), float(d["m0"]), 0)
        vol = qb.lib().b200_volume()
        if "ud" in d:
            qb.upload_ud(d["ud"])
            qb.upload_swd(d["swd"])
        else:
            # the device generator with global site counters: the slab of
            # the single-rank field
            qb.random_ud(float(d["eps"]), int(d["seed"]))
            res["ud_gen"] = qb.download_ud(vol)
            # the SW term from the links, the clover leaves of the boundary
            # planes with the neighbours' links
            qb.sw_term()
            res["sw_gen"] = qb.download_swd(vol)
        res["ud_back"] = qb.download_ud(vol)
        mu = float(d["mu"])
        s, r0 = d["s"], d["r0"]
        res["Dw_dble"] = qb.dirac_ref("Dw", 64, mu, s)
        res["Dwhat_dble"] = qb.dirac_ref("Dwhat", 64, mu, s, r0)
        res["Dwoe_dble"] = qb.dirac_ref("Dwoe", 64, mu, s, r0)
        res["Dw"] = qb.dirac_ref("Dw", 32, mu, s.astype(np.float32))
        res["Dwhat"] = qb.dirac_ref("Dwhat", 32, mu, s.astype(np.float32), r0.astype(np.float32))
        qb.set_sap_parms(bs, 1, 4, 1)
        qb.set_sap_variant(int(d["variant"]))
        psi, rho = qb.sap_ref(mu, 1, 4, np.zeros_like(s, dtype=np.float32), s.astype(np.float32))
        res["sap_psi"], res["sap_rho"] = psi, rho
        qb.set_sap_parms(bs, 1, 4, 5)
        psi, rho_n, ifail, status = qb.sap_gcr(16, 256, 0, 1e-10, mu, s)
        res["gcr_psi"] = psi
        res["gcr"] = np.array([rho_n, ifail, status])
        res["nexchange"] = np.array([qb.dd_info()[3]])
        qb.release_workspace()
        qb.dd_off()
    except Exception as e:                      # reported to the parent
        res["error"] = np.array([repr(e)])
    finally:
        dist.destroy_process_group()
    np.savez(outp % rank, **res)
