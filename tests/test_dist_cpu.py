"""The multi-rank logic of bench.py on CPU: two gloo ranks (127.0.0.1)
synchronise, reduce their step times to the maximum over ranks (the value
every rank then reports), and the reference arm runs on rank 0 only (the
other ranks return 0 without work)."""
import multiprocessing as mp
import os
import socket
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench

    d = bench.Dist()
    try:
        d.barrier()
        m = d.max(1.5 * (rank + 1))

        class A:
            gpus, steps, warmup = world, 1, 3

        rc = bench.run_reference(A(), d) if rank != 0 else 0
        q.put((rank, d.world, m, rc))
    finally:
        d.close()


def test_two_gloo_ranks():
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[0] for o in out] == [0, 1]
    assert all(o[1] == 2 for o in out)
    assert all(o[2] == 3.0 for o in out)          # max over ranks of 1.5 and 3.0
    assert out[1][3] == 0                          # reference arm: rank 1 does no work
