"""The plan of the host pipeline of Dw / Dw_dble (pieces: the thinnest
x0-slabs of at least 131072 sites, or a sixteenth of the lattice, whose
sites are one contiguous range of each parity half of the storage order;
slabs: the block rows along x0), computed by the library's host code
without a device, against a plain restatement here, and a simulation of
the pipeline's schedule (the order in which pieces are copied in, block
rows are launched and pieces are copied out) that checks every row runs
after the pieces holding its planes and neighbour planes are in and every
piece goes out once, after its own input and all its rows."""
import numpy as np
import pytest

import openqcd_b200 as qb

MIN_SITES = 131072


def plan(L, bs, ipt):
    """(P, pieces, rows) or None: the restatement of the plan"""
    L0, vol = L[0], int(np.prod(L))
    ps = vol // L0
    if L0 // bs[0] < 3:
        return None
    x = np.indices(L).reshape(4, -1)
    par = x.sum(axis=0) & 1
    lo = np.full((L0, 2), vol)
    hi = np.full((L0, 2), -1)
    for t in range(L0):
        for p in range(2):
            q = ipt[(x[0] == t) & (par == p)]
            lo[t, p], hi[t, p] = q.min(), q.max()
    for P in range(1, L0 // 3 + 1):
        if L0 % P or P * ps < min(MIN_SITES, vol // 16):
            continue
        ok = all(hi[i:i + P, p].max() - lo[i:i + P, p].min() + 1 == P * ps // 2
                 for i in range(0, L0, P) for p in range(2))
        if ok:
            return P, [(i, i + P) for i in range(0, L0, P)], [(k * bs[0], (k + 1) * bs[0]) for k in range(L0 // bs[0])]
    return None


def schedule(L0, P, pieces, rows):
    """the pipeline's schedule as the library issues it; asserts its
    ordering rules and returns the transfer position after which each row
    runs"""
    npc = len(pieces)

    def pos(i):
        return 0 if i == npc - 1 else i + 1

    need = [max(pos(((t + L0) % L0) // P) for t in range(r[0] - 1, r[1] + 1)) for r in rows]
    left = [0] * npc
    for r in rows:
        for i in range(r[0] // P, (r[1] - 1) // P + 1):
            left[i] += 1
    arrived, ran, out = set(), [], []
    for j in range(npc):
        arrived.add(npc - 1 if j == 0 else j - 1)
        for k, r in enumerate(rows):
            if need[k] != j:
                continue
            assert all(((t + L0) % L0) // P in arrived for t in range(r[0] - 1, r[1] + 1))
            ran.append(k)
            for i in range(r[0] // P, (r[1] - 1) // P + 1):
                left[i] -= 1
                if left[i] == 0:
                    assert i in arrived
                    out.append(i)
    assert sorted(ran) == list(range(len(rows)))
    assert sorted(out) == list(range(npc))
    return need


CASES = [((16, 8, 8, 8), (4, 4, 4, 4), 16, 4), ((16, 8, 8, 8), (2, 4, 4, 4), 16, 8),
         ((64, 32, 32, 32), (4, 4, 4, 4), 16, 16), ((96, 48, 48, 48), (6, 6, 6, 6), 48, 16),
         ((8, 8, 8, 8), (2, 4, 4, 4), 8, 4), ((8, 8, 8, 8), (4, 4, 4, 4), 0, 0)]


@pytest.mark.parametrize("L,bs,npc,nsl", CASES)
def test_plan_lexicographic(L, bs, npc, nsl):
    ipt = qb.even_first_ipt(L)
    assert qb.pipeline_plan(L, bs, ipt) == (npc, nsl)
    r = plan(L, bs, ipt)
    if npc == 0:
        assert r is None
        return
    P, pieces, rows = r
    assert (len(pieces), len(rows)) == (npc, nsl)
    schedule(L[0], P, pieces, rows)


def test_plan_reference_ipt():
    """the reference build's ipt (16 threads: L0_TRD = 4): pieces of four
    planes; with blocks two planes thick every piece spans two rows"""
    import reflib
    L = (16, 8, 8, 8)
    if not reflib.available(L):
        pytest.skip("reference oracle library not built")
    r = reflib.RefLib(L)
    r.init()
    ipt = r.ipt()
    for bs, nsl in (((4, 4, 4, 4), 4), ((2, 4, 4, 4), 8)):
        assert qb.pipeline_plan(L, bs, ipt) == (4, nsl)
        P, pieces, rows = plan(L, bs, ipt)
        assert P == 4
        schedule(L[0], P, pieces, rows)


def test_plan_needs_contiguous_pieces():
    """an even-first order that scatters the planes: no pipeline"""
    L = (16, 8, 8, 8)
    x = np.indices(L).reshape(4, -1)
    par = x.sum(axis=0) & 1
    rng = np.random.default_rng(3)
    ipt = np.empty(par.size, dtype=np.int32)
    for p in range(2):
        idx = np.nonzero(par == p)[0]
        ipt[idx] = p * (par.size // 2) + rng.permutation(idx.size)
    assert qb.pipeline_plan(L, (4, 4, 4, 4), ipt) == (0, 0)


def test_plan_rejects_bad_blocks():
    with pytest.raises(qb.B200Error):
        qb.pipeline_plan((16, 8, 8, 8), (3, 4, 4, 4), qb.even_first_ipt((16, 8, 8, 8)))
