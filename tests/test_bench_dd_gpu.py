"""bench.py with two ranks along x0 (torchrun, 127.0.0.1), faces through the
host (--dd-transport host, gloo), both ranks on the one GPU of the machine:
the sharded-lattice mode runs the Dw_dble timing and prints one JSON line
from rank 0 with n_gpus = 2 and the aggregate value.  (NCCL between ranks
needs a GPU per rank.)"""
import json
import os
import socket
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_bench_two_ranks_host_transport():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(_free_port()), os.path.join(ROOT, "bench.py"), "--gpus", "2",
           "--dd-transport", "host", "--steps", "3", "--warmup", "3", "--lattice", "16,8,8,8", "--no-cpu-baseline",
           "--no-solver", "--no-e2e"]
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-4000:]
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, p.stdout
    out = json.loads(lines[0])
    assert out["n_gpus"] == 2 and out["value"] > 0 and out["steps"] == 3
