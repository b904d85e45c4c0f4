"""Data-parallel training of the learned preconditioner, host side, on CPU:
two gloo ranks (127.0.0.1) each hold their own training pairs on their own
gauge field and run openqcd_b200.data_parallel_steps with the gradients of
the network's CPU oracle (oracle/ptnet.py: the loss and weight packing of
the device kernels) and an Adam step; loss and gradients are summed over
the ranks and divided by their number.  Both ranks end with the same
weights, equal to those of one process that averages the two ranks'
minibatch gradients itself."""
import multiprocessing as mp
import os
import socket
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
L = (4, 4, 4, 4)
STEPS, BATCH, LR, NPAIRS = 3, 2, 1e-2, 4


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _paths():
    for p in (os.path.join(ROOT, "openqcd-2.4.2_b200"), os.path.join(ROOT, "oracle")):
        if p not in sys.path:
            sys.path.insert(0, p)


def _rank_data(rank):
    """this rank's gauge field and training pairs"""
    import ptnet
    rng = np.random.default_rng(100 + rank)
    U = ptnet.random_links(L, rng)
    V = int(np.prod(L))
    pairs = [(rng.standard_normal((V, 4, 3)) + 1j * rng.standard_normal((V, 4, 3)),
              rng.standard_normal((V, 4, 3)) + 1j * rng.standard_normal((V, 4, 3))) for _ in range(NPAIRS)]
    return U, ptnet.neighbours(L), pairs


def _w0():
    import ptnet
    rng = np.random.default_rng(7)
    n = sum(2 * 9 * ptnet.CH[l] * ptnet.CH[l + 1] for l in range(3))
    return 0.1 * rng.standard_normal(n)


class _Adam:
    def __init__(self, w):
        self.w, self.m, self.v, self.t = w.copy(), np.zeros_like(w), np.zeros_like(w), 0

    def step(self, g, lr):
        g = np.asarray(g, dtype=np.float64)
        self.t += 1
        self.m = 0.9 * self.m + 0.1 * g
        self.v = 0.999 * self.v + 0.001 * g * g
        self.w -= lr * (self.m / (1 - 0.9 ** self.t)) / (np.sqrt(self.v / (1 - 0.999 ** self.t)) + 1e-8)


def _grad_fn(data, opt):
    import ptnet
    U, nb, pairs = data

    def fn(idx):
        Ws = ptnet.unpack(opt.w)
        out = [ptnet.loss_grad(U, nb, Ws, pairs[i][0], pairs[i][1]) for i in idx]
        return sum(o[0] for o in out) / len(idx), sum(o[1] for o in out) / len(idx)
    return fn


def _rank(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    _paths()
    import torch
    import torch.distributed as dist
    import openqcd_b200 as qb

    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        opt = _Adam(_w0())

        def allreduce(v):
            t = torch.from_numpy(np.ascontiguousarray(v))
            dist.all_reduce(t, op=dist.ReduceOp.SUM)
            return t.numpy()

        hist = qb.data_parallel_steps(_grad_fn(_rank_data(rank), opt), opt.step, NPAIRS, STEPS, BATCH, LR,
                                      11 + rank, allreduce, world)
        q.put((rank, opt.w, hist))
    finally:
        dist.destroy_process_group()


def test_data_parallel_training_two_gloo_ranks():
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=300) for _ in procs), key=lambda o: o[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert np.array_equal(out[0][1], out[1][1])          # the ranks agree
    assert out[0][2] == out[1][2]

    # one process averaging the two ranks' minibatch gradients itself
    _paths()
    opt = _Adam(_w0())
    fns = [_grad_fn(_rank_data(r), opt) for r in range(2)]
    rngs = [np.random.default_rng(11 + r) for r in range(2)]
    hist = []
    for _ in range(STEPS):
        bufs = []
        for r in range(2):
            loss, g = fns[r](rngs[r].integers(0, NPAIRS, size=BATCH))
            bufs.append(np.concatenate([[loss], np.asarray(g, dtype=np.float64)]))
        buf = (bufs[0] + bufs[1]) / 2
        opt.step(buf[1:].astype(np.float32), LR)
        hist.append(float(buf[0]))
    assert np.allclose(out[0][1], opt.w, rtol=0, atol=1e-12)
    assert np.allclose(out[0][2], hist, rtol=1e-12)
    assert not np.allclose(opt.w, _w0())                 # the weights moved
