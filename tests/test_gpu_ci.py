"""GPU parity of the CI side (RDMs, regularised inverse, one-body matrix
elements, assembled sparse matrices, sigma) against the oracle, through the C ABI."""
import numpy as np
import pytest

from oracle import sinc_oracle as orc
from oracle.walks_oracle import CIWalks

pytestmark = pytest.mark.gpu
TOL = 1e-11


def relerr(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


def seeded_avector(nc, seed):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal(nc) + 1j * rng.standard_normal(nc)
    return a / np.linalg.norm(a)


@pytest.fixture(scope="module", params=[(2, 0), (4, 0), (3, 1)], ids=["2e", "4e", "3e"])
def setup(request, built_lib):
    from sincgpu import SincProject, WalkTables
    numelec, ms = request.param
    n = 5
    sysm = orc.SincSystem(21, 0.4, [[0, 0, 0]], [2.0])
    gpu = SincProject(21, 0.4, [[0, 0, 0]], [2.0], n)
    walks = WalkTables(numelec, n, ms)
    gpu.ci_attach(walks)
    ow = CIWalks(numelec, n, ms)
    phi = orc.seeded_orbitals(sysm, n, seed=21)
    a = seeded_avector(ow.numconfig, seed=22)
    yield sysm, gpu, ow, phi, a
    gpu.close()


def test_denmat_and_inverse(setup):
    sysm, gpu, ow, phi, a = setup
    den_ref = ow.getdenmat00(a)
    inv_ref = orc.invmatsmooth(den_ref)
    den, inv = gpu.getdenmat(a)
    assert relerr(den, den_ref) < TOL
    assert relerr(inv, inv_ref) < 1e-10
    assert relerr(den @ inv, np.eye(5)) < 1e-10


@pytest.mark.parametrize("eps", [0.0, 1e-7])
def test_regularised_inverse_near_singular(setup, eps):
    """A nearly single-determinant A-vector leaves orbitals (almost) empty: the
    density matrix is (nearly) singular and the denreg regularisation of
    invmatsmooth decides the inverse (MCTDH.SRC/utils.f90:578-591)."""
    sysm, gpu, ow, phi, a = setup
    b = np.zeros(ow.numconfig, dtype=np.complex128)
    b[0] = 1.0
    b = b + eps * a
    b /= np.linalg.norm(b)
    den_ref = ow.getdenmat00(b)
    inv_ref = orc.invmatsmooth(den_ref)
    den, inv = gpu.getdenmat(b)
    assert relerr(den, den_ref) < TOL
    assert relerr(inv, inv_ref) < 1e-8


def test_tworeducedx(setup):
    sysm, gpu, ow, phi, a = setup
    t_ref = ow.get_tworeducedx(a)
    assert relerr(gpu.get_tworeducedx(a), t_ref) < TOL
    b = seeded_avector(ow.numconfig, seed=23)
    assert relerr(gpu.get_tworeducedx(a, b), ow.get_tworeducedx(a, b)) < TOL


def test_onebody_matel(setup):
    sysm, gpu, ow, phi, a = setup
    pot, ke, z = gpu.onebody_matel(phi)
    ph = np.conj(phi).T
    assert relerr(pot, ph @ sysm.mult_pot(phi)) < TOL
    assert relerr(ke, ph @ sysm.mult_ke(phi)) < TOL
    assert relerr(z, ph @ sysm.mult_zdipole(phi)) < TOL


@pytest.mark.parametrize("ez", [0.0, 0.03])
def test_sigma(setup, ez):
    sysm, gpu, ow, phi, a = setup
    mat, _ = sysm.call_twoe_matel00(phi, phi)
    ph = np.conj(phi).T
    pot = ph @ sysm.mult_pot(phi)
    ke = ph @ sysm.mult_ke(phi)
    z = ph @ sysm.mult_zdipole(phi)
    gpu.assemble_sparsemats(mat, pot, ke, z)
    xpot = ow.assemble_doubles(mat)
    xone = ow.assemble_singles(pot)
    xop = ow.assemble_singles(ke)
    nucdip = float(np.sum(sysm.nuccharges * sysm.centershift[:, 2] / 2.0 * sysm.spacing))
    xz = ow.assemble_singles(z) * ez if ez else None
    ref = ow.sparsesparsemult(a, xpot, xone, xop, constant=sysm.nucrepulsion + ez * nucdip, xpulse=xz)
    out = gpu.sparseconfigmult(a, ezfield=ez)
    assert relerr(out, ref) < TOL


def test_energy_from_sigma_equals_energy_from_rdms(setup):
    """<A|H|A> through the sigma product equals the RDM contraction
    sum h(a,b) den(b,a) + 1/2 sum twoematel tally + nucrepulsion."""
    sysm, gpu, ow, phi, a = setup
    mat, _ = sysm.call_twoe_matel00(phi, phi)
    ph = np.conj(phi).T
    pot = ph @ sysm.mult_pot(phi)
    ke = ph @ sysm.mult_ke(phi)
    z = ph @ sysm.mult_zdipole(phi)
    gpu.assemble_sparsemats(mat, pot, ke, z)
    e_sigma = np.vdot(a, gpu.sparseconfigmult(a))
    den, _ = gpu.getdenmat(a)
    tally = gpu.get_tworeducedx(a)
    e_rdm = np.sum((pot + ke) * den.T) + 0.5 * np.sum(mat * tally) + sysm.nucrepulsion
    assert abs(e_sigma - e_rdm) < 1e-10 * abs(e_rdm)


def test_dipole_z(setup):
    from oracle.walks_oracle import dipole_z
    sysm, gpu, ow, phi, a = setup
    mat, _ = sysm.call_twoe_matel00(phi, phi)
    ph = np.conj(phi).T
    pot, ke, z = ph @ sysm.mult_pot(phi), ph @ sysm.mult_ke(phi), ph @ sysm.mult_zdipole(phi)
    gpu.assemble_sparsemats(mat, pot, ke, z)
    nucdip = float(np.sum(sysm.nuccharges * sysm.centershift[:, 2] / 2.0 * sysm.spacing))
    d_ref, n_ref = dipole_z(ow, ow.assemble_singles(z), a, nucdip)
    d, nn = gpu.dipole_z(a)
    assert abs(d - d_ref) < TOL * max(abs(d_ref), 1.0)
    assert nn == pytest.approx(n_ref, rel=1e-14)
    # the expectation of a hermitian operator is real
    assert abs(d.imag) < 1e-12 * max(abs(d), 1.0)
