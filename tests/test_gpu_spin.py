"""Spin projection (basis_project, allspinproject=1) on the GPU against the
oracle, and its commutation with the spin-free CI Hamiltonian.  Tolerance 1e-13
(the projection is one small real matrix-vector product per spin set)."""
import numpy as np
import pytest

from oracle import sinc_oracle as orc
from oracle.walks_oracle import CIWalks, SpinSets

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=[(2, 0, 0), (3, 1, 1), (4, 0, 0), (4, 0, 2), (4, 2, 2)],
                ids=["2e-S0", "3e-S1/2", "4e-S0", "4e-S1-ms0", "4e-S1-ms1"])
def spin(request, built_lib):
    from sincgpu import SincProject, WalkTables
    numelec, ms, two_s = request.param
    n = 5
    sysm = orc.SincSystem(15, 0.5, [[0, 0, 0]], [2.0], toothnbig=40, toothnsmall=10)
    gpu = SincProject(15, 0.5, [[0, 0, 0]], [2.0], n, toothnbig=40, toothnsmall=10)
    gpu.ci_attach(WalkTables(numelec, n, ms).build_spin(two_s))
    ow = CIWalks(numelec, n, ms)
    sp = SpinSets(ow, two_s)
    yield sysm, gpu, ow, sp
    gpu.close()


def test_spin_project_matches_oracle(spin):
    _, gpu, ow, sp = spin
    rng = np.random.default_rng(81)
    a = rng.standard_normal(ow.numconfig) + 1j * rng.standard_normal(ow.numconfig)
    out = gpu.spin_project(a)
    ref = sp.project(a)
    assert np.abs(out - ref).max() < 1e-13
    assert np.abs(gpu.spin_project(out) - out).max() < 1e-13      # idempotent


def test_sigma_commutes_with_spin_projection(spin):
    """H is spin free: P H P a = H P a, so sigma keeps a spin eigenstate in its space."""
    sysm, gpu, ow, sp = spin
    n = 5
    phi = orc.seeded_orbitals(sysm, n, seed=82)
    mat, _ = sysm.call_twoe_matel00(phi, phi)
    ph = np.conj(phi).T
    pot, ke, z = ph @ sysm.mult_pot(phi), ph @ sysm.mult_ke(phi), ph @ sysm.mult_zdipole(phi)
    gpu.assemble_sparsemats(mat, pot, ke, z)
    rng = np.random.default_rng(83)
    a = rng.standard_normal(ow.numconfig) + 1j * rng.standard_normal(ow.numconfig)
    pa = gpu.spin_project(a)
    hpa = gpu.sparseconfigmult(pa)
    assert np.abs(gpu.spin_project(hpa) - hpa).max() < 1e-11 * np.abs(hpa).max()
