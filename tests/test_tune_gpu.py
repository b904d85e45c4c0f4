"""The block-shape autotuner (b200_tune_block_shape, no reference
counterpart): every candidate SAP block shape that fits the lattice is
scored by the residual reduction per second of a few SAP+GCR steps; shapes
that do not fit score -1; the best one stays in force with the same fields,
so the operators still equal the reference's and sap_gcr still converges."""
import numpy as np
import pytest

import openqcd_b200 as qb
from helpers import Setup, site_rel_err

pytestmark = pytest.mark.gpu

L = (16, 8, 8, 8)


def test_block_shape_tuner():
    st = Setup(L, (4, 4, 4, 4), eps=0.4, csw=1.7, m0=-0.05)
    qb.set_sap_parms((4, 4, 4, 4), 1, 4, 5)
    cands = [(4, 4, 4, 4), (8, 4, 4, 4), (4, 4, 4, 8), (6, 6, 6, 6)]
    best, scores = qb.tune_block_shape(cands, nsteps=6, mu=0.0, Ns=0)
    print("block shapes", cands, "scores", scores, "best", best)
    assert scores[2] == -1.0 and scores[3] == -1.0          # 8 / 8 = 1 block along x3; 6 does not divide 8
    assert scores[0] > 0 and scores[1] > 0
    assert best == cands[int(np.argmax(scores))]
    s = st.source(3)
    r_ref = st.ref.dirac_dble(0, 0.1, s)
    assert site_rel_err(qb.dirac_ref("Dw", 64, 0.1, s), r_ref, st.vol) <= 1e-13
    psi, rho, ifail, status = qb.sap_gcr(16, 256, 0, 1e-10, 0.0, s)
    r = s - st.ref.dirac_dble(0, 0.0, psi)
    assert ifail == 0 and np.linalg.norm(r) / np.linalg.norm(s) <= 1.5e-10


def test_block_shape_tuner_deflated():
    """the deflated objective: every fitting candidate gets its own subspace
    and a positive score; the deflated solver then runs on the best shape"""
    st = Setup(L, (4, 4, 4, 4), eps=0.4, csw=1.7, m0=-0.05)
    qb.set_sap_parms((4, 4, 4, 4), 1, 4, 5)
    qb.set_dfl_pro_parms(16, 256, 1e-2, 24, 1e-2)
    qb.set_dfl_gen_parms(1.0 / (2.0 * (4.0 - 0.05)), 0.0, 5, 4, 4)
    cands = [(4, 4, 4, 4), (8, 4, 4, 4), (4, 4, 4, 8)]
    best, scores = qb.tune_block_shape(cands, nsteps=4, mu=0.0, Ns=8)
    print("deflated: scores", scores, "best", best)
    assert scores[0] > 0 and scores[1] > 0 and scores[2] == -1.0
    qb.set_dfl_parms(best, 8)
    f, _ = qb.dfl_modes(1)
    assert f == 0
    s = st.source(5)
    psi, rho, ifail, status = qb.dfl_sap_gcr(16, 256, 0, 1e-10, 0.0, s)
    r = s - st.ref.dirac_dble(0, 0.0, psi)
    assert ifail == 0 and np.linalg.norm(r) / np.linalg.norm(s) <= 1.5e-10
