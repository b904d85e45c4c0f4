"""Data-parallel training of the learned preconditioner on the device: the
minibatch gradient is the mean of the per-pair gradients, the Adam step
with a given gradient moves the weights as Adam's first step does, and two
ranks (processes on this GPU with gloo; the host sums the gradients between
kernel launches, no kernel waits on another) that train on pairs from their
own gauge fields end with identical weights."""
import multiprocessing as mp
import os
import socket
import sys

import numpy as np
import pytest

import openqcd_b200 as qb
from helpers import Setup

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
L = (8, 8, 8, 8)
BS = (4, 4, 4, 4)


@pytest.fixture(scope="module")
def pairs():
    s = Setup(L, BS, eps=0.4, csw=1.5, m0=-0.2)
    qb.set_sap_parms(BS, 1, 4, 5)
    rs = [qb.DevField(32) for _ in range(3)]
    es = [qb.DevField(32) for _ in range(3)]
    qb.net_make_pairs(rs, es, 0.0, 1e-6, seed=3)
    qb.net_init(1, 0.25)
    yield s, rs, es
    for f in rs + es:
        f.free()


def test_batch_grad_is_mean(pairs):
    _, rs, es = pairs
    one = [qb.net_grad(r, e) for r, e in zip(rs, es)]
    loss, g = qb.net_batch_grad(rs, es)
    gm = sum(o[1].astype(np.float64) for o in one) / 3
    assert abs(loss - sum(o[0] for o in one) / 3) <= 1e-6 * loss
    assert np.linalg.norm(g - gm) <= 1e-5 * np.linalg.norm(gm)


def test_adam_first_step(pairs):
    """After net_set_weights the Adam state is fresh: the first step moves
    each weight by lr g / (|g| + 1e-8)."""
    _, rs, es = pairs
    w0 = qb.net_get_weights()
    qb.net_set_weights(w0)
    _, g = qb.net_batch_grad(rs, es)
    lr = 1e-3
    qb.net_adam_step(g, lr)
    w1 = qb.net_get_weights()
    want = w0 - lr * g / (np.abs(g) + 1e-8)
    assert np.abs(w1 - want).max() <= 1e-6
    qb.net_set_weights(w0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, os.path.join(ROOT, "openqcd-2.4.2_b200"))
    import torch.distributed as dist
    import openqcd_b200 as qbr

    qbr.set_device(0)
    qbr.geometry(L, BS, qbr.even_first_ipt(L))
    qbr.set_parms(1.5, -0.2, 0)
    qbr.random_ud(0.4, 100 + rank)             # each rank its own gauge field
    qbr.sw_term()
    qbr.set_sap_parms(BS, 1, 4, 5)
    rs = [qbr.DevField(32) for _ in range(4)]
    es = [qbr.DevField(32) for _ in range(4)]
    qbr.net_make_pairs(rs, es, 0.0, 1e-6, seed=9 + rank)
    qbr.net_init(1, 0.25)                      # the same initial weights
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        hist = qbr.net_train_data_parallel(rs, es, 4, 2, 3e-3, seed=5)
        q.put((rank, qbr.net_get_weights(), hist))
    finally:
        dist.destroy_process_group()


def test_two_ranks_identical_weights():
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=600) for _ in procs), key=lambda o: o[0])
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert np.array_equal(out[0][1], out[1][1])
    assert out[0][2] == out[1][2] and all(np.isfinite(out[0][2]))
