"""Configuration and spinor-field files in the universal format
(modules/archive/archive.c:804-977, sarchive.c:424-620) against the
reference's own export/import on the same fields: the link and spinor
payloads must be byte-identical, the header plaquette and square norm equal
to 1e-13, and each side must read the other's files back exactly."""
import os

import numpy as np
import pytest

import openqcd_b200 as qb
from helpers import Setup

pytestmark = pytest.mark.gpu

L = (8, 8, 8, 8)


@pytest.fixture(scope="module")
def setup():
    return Setup(L, (4, 4, 4, 4), eps=0.4, csw=1.5, m0=0.0)


def split(path, nint):
    b = open(path, "rb").read()
    hdr = np.frombuffer(b[:4 * nint], dtype=np.int32)
    val = np.frombuffer(b[4 * nint:4 * nint + 8], dtype=np.float64)[0]
    return hdr, val, b[4 * nint + 8:]


def test_plaquette(setup):
    ref = setup.ref.plaq_sum()
    assert abs(qb.plaq_sum() - ref) <= 1e-13 * abs(ref)


def test_export_cnfg_matches_reference(setup, tmp_path):
    a, b = str(tmp_path / "ref.cnfg"), str(tmp_path / "dev.cnfg")
    setup.ref.export_cnfg(a)
    qb.export_cnfg(b)
    ha, pa, la = split(a, 4)
    hb, pb, lb = split(b, 4)
    assert list(ha) == list(hb) == list(L)
    assert abs(pa - pb) <= 1e-13 * abs(pa)
    assert la == lb


def test_import_cnfg(setup, tmp_path):
    a = str(tmp_path / "ref.cnfg")
    setup.ref.export_cnfg(a)
    qb.random_ud(0.3, 99)                 # overwrite the device field
    qb.import_cnfg(a)
    assert np.array_equal(qb.download_ud(setup.vol), setup.ud)
    with pytest.raises(qb.B200Error):     # the SW term is stale after an import
        qb.dirac_ref("Dw", 64, 0.0, setup.source(1))
    qb.upload_swd(setup.swd)
    # and the reference reads the library's file back to the same field
    b = str(tmp_path / "dev.cnfg")
    qb.export_cnfg(b)
    setup.ref.gen_links(0.2, 7)
    setup.ref.import_cnfg(b)
    assert np.array_equal(setup.ref.ud(), setup.ud)
    setup.ref.set_ud(setup.ud)


@pytest.mark.parametrize("eo", [0, 1])
def test_sfld(setup, tmp_path, eo):
    sd = setup.source(5)
    a, b = str(tmp_path / "ref.sfld"), str(tmp_path / "dev.sfld")
    setup.ref.export_sfld(a, eo, sd)
    qb.export_sfld(b, eo, sd)
    ha, na, pa = split(a, 5)
    hb, nb, pb = split(b, 5)
    assert list(ha) == list(hb) == list(L) + [eo]
    assert abs(na - nb) <= 1e-13 * na
    assert pa == pb
    back = qb.import_sfld(a, eo, np.zeros_like(sd))
    n = setup.vol // 2 if eo else setup.vol
    assert np.array_equal(back.reshape(-1, 24)[:n], sd.reshape(-1, 24)[:n])
    assert np.array_equal(setup.ref.import_sfld(b, eo).reshape(-1, 24)[:n], sd.reshape(-1, 24)[:n])


def test_import_errors(setup, tmp_path):
    bad = str(tmp_path / "bad.cnfg")
    with open(bad, "wb") as f:
        f.write(np.array([4, 4, 4, 4], dtype=np.int32).tobytes() + np.array([3.0]).tobytes())
    with pytest.raises(qb.B200Error):
        qb.import_cnfg(bad)
    with pytest.raises(qb.B200Error):
        qb.import_cnfg(str(tmp_path / "missing.cnfg"))
