"""Phase angles theta of the spatial boundary conditions (set_bc_parms,
modules/flags/lat_parms.c:516; set_ud_phase, modules/uflds/uflds.c:249-355):
the reference multiplies U(x,k) by exp(i theta[k-1]/N[k]), so the links are
U(3), not SU(3).  The device operators read the phased links as given, the
SW term is unchanged by the phases (every clover leaf is a closed loop), the
SAP block solver falls back from its 12-real link reads to the 18-real ones
(the SU(3) check fails), and fields made on the device or read from files
carry the phase of the reference."""
import numpy as np
import pytest

import openqcd_b200 as qb
from helpers import Setup, rel_norm_err, site_rel_err

pytestmark = pytest.mark.gpu

L = (8, 8, 8, 8)
BS = (4, 4, 4, 4)
THETA = (0.5, -0.8, 1.3)
MU = 0.05


@pytest.fixture(scope="module")
def setup():
    s = Setup(L, BS, eps=0.4, csw=1.5, m0=-0.1, theta=THETA)
    yield s
    qb.set_bc_theta((0.0, 0.0, 0.0))


def test_phased_links_are_u3(setup):
    """The reference's links carry the phase: U(x,1) exp(-i theta[0]/N1) is
    SU(3) (det 1) while U(x,1) itself is not."""
    ud = setup.ud.reshape(setup.vol // 2, 8, 3, 3, 2)
    u = ud[..., 0] + 1j * ud[..., 1]
    ph = np.exp(1j * THETA[0] / L[1])
    det = np.linalg.det(u[:, 2])                    # direction 1, forward
    assert np.abs(det - ph ** 3).max() < 1e-12
    assert np.abs(np.linalg.det(u[:, 2] / ph) - 1.0).max() < 1e-12


@pytest.mark.parametrize("op", ["Dw", "Dwee", "Dwoo", "Dwoe", "Dweo", "Dwhat"])
def test_dirac_dble_theta(setup, op):
    s = setup.source(5)
    if op == "Dwhat":
        setup.ref.sw_term(2)       # the reference's Dwhat needs the odd SW term inverted
    ref = setup.ref.dirac_dble(["Dw", "Dwee", "Dwoo", "Dwoe", "Dweo", "Dwhat"].index(op), MU, s)
    if op == "Dwhat":
        setup.ref.sw_term(0)
    out = qb.dirac_ref(op, 64, MU, s)
    assert site_rel_err(out, ref, setup.vol) <= 1e-13


def test_sw_term_theta(setup):
    """The device SW term from the phased links equals the reference's
    (1e-14 per Pauli matrix, as without phases)."""
    assert qb.sw_term() == 0
    a = qb.download_swd(setup.vol, 0).reshape(-1, 36)
    b = setup.swd.reshape(-1, 36)
    assert float((np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)).max()) <= 1e-14
    qb.upload_swd(setup.swd)


def test_sap_gcr_theta(setup):
    """sap_gcr on the phased field reaches the residual in the reference's
    number of steps; the SAP block solver uses the 18-real links."""
    qb.set_sap_parms(BS, 1, 4, 5)
    setup.ref.set_sap_parms(BS, 1, 4, 5)
    eta = setup.source(7)
    psi, rho, ifail, st = qb.sap_gcr(16, 256, 0, 1e-10, MU, eta)
    rpsi, rrho, rifail, rst = setup.ref.sap_gcr(16, 256, 0, 1e-10, MU, eta)
    assert ifail == 0 and rifail == 0
    assert abs(st - rst) <= 1, (st, rst)
    assert rel_norm_err(psi, rpsi) <= 1e-8
    r = eta - setup.ref.dirac_dble(0, MU, psi)
    assert np.linalg.norm(r) / np.linalg.norm(eta) <= 1.5e-10


def test_cnfg_files_theta(setup, tmp_path):
    """export_cnfg takes the phase off (the file holds the same links as
    the reference's file, to rounding) and import_cnfg puts it back."""
    fr = str(tmp_path / "ref_cnfg")
    fd = str(tmp_path / "dev_cnfg")
    setup.ref.export_cnfg(fr)
    qb.upload_ud(setup.ud)
    qb.export_cnfg(fd)
    a = np.fromfile(fr, dtype=np.float64, offset=24)   # 4 int32 sizes, the plaquette, the links
    b = np.fromfile(fd, dtype=np.float64, offset=24)
    assert a.shape == b.shape and np.abs(a - b).max() <= 1e-15
    pa = np.fromfile(fr, dtype=np.float64, count=1, offset=16)[0]
    assert abs(pa - np.fromfile(fd, dtype=np.float64, count=1, offset=16)[0]) <= 1e-13
    qb.import_cnfg(fr, 0)
    assert np.abs(qb.download_ud(setup.vol) - setup.ud).max() <= 1e-15
    # the reference reads the library's file back to its phased field
    setup.ref.import_cnfg(fd)
    assert np.abs(setup.ref.ud() - setup.ud).max() <= 1e-15
    setup.ref.set_ud(setup.ud)
    qb.upload_ud(setup.ud)
    qb.upload_swd(setup.swd)


def test_random_ud_theta(setup):
    """Fields made on the device carry the phase: the spatial links divided
    by exp(i theta[k-1]/N[k]) are SU(3)."""
    qb.random_ud(0.3, 99)
    u = qb.download_ud(setup.vol).reshape(setup.vol // 2, 8, 3, 3, 2)
    u = u[..., 0] + 1j * u[..., 1]
    for k in range(3):
        ph = np.exp(1j * THETA[k] / L[k + 1])
        v = u[:, 2 + 2 * k] / ph
        assert np.abs(np.linalg.det(v) - 1.0).max() < 1e-12
        assert np.abs(np.einsum("nij,nkj->nik", v, v.conj()) - np.eye(3)).max() < 1e-12
    qb.upload_ud(setup.ud)
    qb.upload_swd(setup.swd)
