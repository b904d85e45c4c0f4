"""The SAP preconditioner as a CUDA graph: sap_gcr with graphs on and off
runs the same kernels on the same data in the same order, so the solutions
are identical and so are the iteration counts; the graph is captured once
per parameter set and replayed at every GCR step and by later solves."""
import numpy as np
import pytest

import openqcd_b200 as qb
from helpers import Setup

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    s = Setup((8, 8, 8, 8), (4, 4, 4, 4), eps=0.4, csw=1.5, m0=-0.05)
    qb.set_sap_parms((4, 4, 4, 4), 1, 4, 5)
    yield s
    qb.set_cuda_graphs(True)


@pytest.mark.parametrize("mu", [0.0, 0.05])
def test_graph_equals_direct(setup, mu):
    eta = setup.source(51)
    prev = qb.set_cuda_graphs(False)
    try:
        psi0, rho0, f0, st0 = qb.sap_gcr(16, 256, 0, 1e-10, mu, eta)
        assert qb.graphs_cached() == 0
        qb.set_cuda_graphs(True)
        psi1, rho1, f1, st1 = qb.sap_gcr(16, 256, 0, 1e-10, mu, eta)
        n1 = qb.graphs_cached()
        psi2, rho2, f2, st2 = qb.sap_gcr(16, 256, 0, 1e-10, mu, eta)
    finally:
        qb.set_cuda_graphs(prev)
    assert f0 == f1 == f2 == 0
    assert st0 == st1 == st2
    assert np.array_equal(psi0, psi1) and np.array_equal(psi1, psi2)
    assert rho0 == rho1 == rho2
    # one graph for the parameter set, reused by the second solve
    assert n1 >= 1 and qb.graphs_cached() == n1


def test_graph_batched(setup):
    """The batched solver without deflation uses the same preconditioner."""
    E = [qb.DevField(64).random(1.0, 60 + i) for i in range(3)]
    out = []
    for on in (False, True):
        qb.set_cuda_graphs(on)
        P = [qb.DevField(64) for _ in E]
        rho, ifail, st, _ = qb.dev_gcr_batch(16, 256, 0, 1e-10, [0.0, 0.02, 0.1], E, P, dfl=False)
        out.append((st, [p.to_ref(setup.vol) for p in P]))
        for p in P:
            p.free()
    qb.set_cuda_graphs(True)
    assert out[0][0] == out[1][0]
    for a, b in zip(out[0][1], out[1][1]):
        assert np.array_equal(a, b)
    for e in E:
        e.free()
