"""Host side of the domain decomposition along x0, on CPU with gloo ranks
(127.0.0.1): the transport openqcd_b200.DomainDecomposition gives the
library, and the library's global double-double sum that every reduction
uses under domain decomposition (modules/utils/qsum.c:389 global_qsum).

- Face exchange: every rank sends its send_dn face to the rank below and its
  send_up face to the rank above (periodic in the rank index); after the
  exchange recv_up holds the upper rank's send_dn and recv_dn the lower
  rank's send_up.  Run with 2 ranks (both neighbours are the same rank, the
  message tags keep the two faces apart) and with 3.
- Global sum: (hi, lo) pairs chosen so that plain double addition loses the
  low parts; the library (b200_dd_global_sum, through the C-to-Python
  all-gather callback) returns the exact sum rounded to double-double, the
  same bits on every rank.
No device work: the buffers are host memory and the copy is a host memmove.
"""
import ctypes
import multiprocessing as mp
import os
import socket
import sys
from fractions import Fraction

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NBYTES = 96 * 64


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _pairs(rank):
    return np.array([1e16 * (rank + 1), 1.0 + rank, 3.0 * (rank + 1), 2.0 ** -60 * (rank + 1)])


def _rank(rank, world, port, q):
    sys.path.insert(0, os.path.join(ROOT, "openqcd-2.4.2_b200"))
    import torch.distributed as dist

    import openqcd_b200 as qb
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        dd = qb.DomainDecomposition(transport="host", memcpy=lambda dst, src, n: ctypes.memmove(dst, src, n))
        dd.install()
        bufs = [np.zeros(NBYTES, dtype=np.uint8) for _ in range(4)]
        bufs[0][:] = (17 * rank + 1) % 251          # send_dn
        bufs[1][:] = (31 * rank + 7) % 251          # send_up
        dd.exchange(*[b.ctypes.data for b in bufs], NBYTES)
        got_up, got_dn = int(bufs[2][0]), int(bufs[3][0])
        uniform = bool((bufs[2] == bufs[2][0]).all() and (bufs[3] == bufs[3][0]).all())
        s = qb.dd_global_sum(_pairs(rank))
        npr = qb.dd_info()[0]
        qb.dd_off()
        q.put((rank, got_up, got_dn, uniform, s.tolist(), npr))
    finally:
        dist.destroy_process_group()


def _run(world):
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return out


def _check(out, world):
    for rank, got_up, got_dn, uniform, s, npr in out:
        assert npr == world
        assert uniform
        assert got_up == (17 * ((rank + 1) % world) + 1) % 251      # the upper rank's send_dn
        assert got_dn == (31 * ((rank - 1) % world) + 7) % 251      # the lower rank's send_up
    sums = [o[4] for o in out]
    assert all(s == sums[0] for s in sums)                          # the same bits on every rank
    for k in range(2):
        exact = sum(Fraction(float(_pairs(r)[2 * k])) + Fraction(float(_pairs(r)[2 * k + 1])) for r in range(world))
        hi, lo = sums[0][2 * k], sums[0][2 * k + 1]
        assert Fraction(hi) + Fraction(lo) == exact or abs(Fraction(hi) + Fraction(lo) - exact) <= abs(exact) * Fraction(1, 2 ** 100)
        assert hi == float(exact)


def test_dd_transport_two_ranks():
    _check(_run(2), 2)


def test_dd_transport_three_ranks():
    _check(_run(3), 3)
