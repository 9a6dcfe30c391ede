"""A-vector Krylov propagation (expoavecprop -> DGEXPVxxx2) on the GPU against
the oracle's restatement of the same Expokit algorithm and against a dense
matrix exponential."""
import numpy as np
import pytest
import scipy.linalg as sl

from oracle import sinc_oracle as orc
from oracle.expokit_oracle import complexify, dgexpv, realify
from oracle.walks_oracle import CIWalks

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=[(2, 0), (4, 0)], ids=["2e", "4e"])
def ci(request, built_lib):
    from sincgpu import SincProject, WalkTables
    numelec, ms = request.param
    n = 5
    sysm = orc.SincSystem(21, 0.4, [[0, 0, 0]], [2.0])
    gpu = SincProject(21, 0.4, [[0, 0, 0]], [2.0], n)
    gpu.ci_attach(WalkTables(numelec, n, ms))
    ow = CIWalks(numelec, n, ms)
    phi = orc.seeded_orbitals(sysm, n, seed=31)
    mat, _ = sysm.call_twoe_matel00(phi, phi)
    ph = np.conj(phi).T
    pot, ke, z = ph @ sysm.mult_pot(phi), ph @ sysm.mult_ke(phi), ph @ sysm.mult_zdipole(phi)
    gpu.assemble_sparsemats(mat, pot, ke, z)
    xp, xo, xk, xz = ow.assemble_doubles(mat), ow.assemble_singles(pot), ow.assemble_singles(ke), ow.assemble_singles(z)

    def sigma(a, ez=0.0):
        return ow.sparsesparsemult(a, xp, xo, xk, constant=sysm.nucrepulsion,
                                   xpulse=(xz * ez if ez else None))

    rng = np.random.default_rng(32)
    a = rng.standard_normal(ow.numconfig) + 1j * rng.standard_normal(ow.numconfig)
    a /= np.linalg.norm(a)
    yield gpu, ow, sigma, a
    gpu.close()


@pytest.mark.parametrize("dt,m,guess", [(0.05, 8, 1.0), (0.05, 6, 0.3), (0.2, 10, 0.25)])
def test_expoavecprop_matches_oracle(ci, dt, m, guess):
    gpu, ow, sigma, a = ci
    tf = -1j * dt                                  # timefac * step, as cmf_prop_avector0 scales it
    mv = lambda x: realify(tf * sigma(complexify(x)))  # noqa: E731
    dot = lambda u, v: float(u @ v)                # noqa: E731
    w_ref, g_ref, info = dgexpv(2 * ow.numconfig, m, 1.0, realify(a), 1e-9, dt, mv, dot, guess,
                                2 * ow.numconfig - 1)
    w, g, nstep = gpu.expoavecprop(a, 1.0, krylovdim=m, tol=1e-9, anorm=dt, stepguess=guess, timefac=tf)
    assert nstep == info["nstep"]
    assert g == pytest.approx(g_ref, rel=1e-12)
    w_ref = complexify(w_ref)
    assert np.abs(w - w_ref).max() < 1e-11
    # and against the dense exponential of the same Hamiltonian
    H = np.column_stack([sigma(e) for e in np.eye(ow.numconfig, dtype=np.complex128)])
    exact = sl.expm(tf * H) @ a
    assert np.abs(w - exact).max() < 1e-7
    assert abs(np.linalg.norm(w) - 1.0) < 1e-8      # unitary propagation


def test_expoavecprop_with_field(ci):
    gpu, ow, sigma, a = ci
    dt, ez = 0.05, 0.02
    tf = -1j * dt
    mv = lambda x: realify(tf * sigma(complexify(x), ez))  # noqa: E731
    w_ref, g_ref, info = dgexpv(2 * ow.numconfig, 8, 1.0, realify(a), 1e-9, dt, mv,
                                lambda u, v: float(u @ v), 1.0, 2 * ow.numconfig - 1)
    w, g, nstep = gpu.expoavecprop(a, 1.0, krylovdim=8, tol=1e-9, anorm=dt, stepguess=1.0, timefac=tf,
                                   ezfield=ez)
    assert nstep == info["nstep"]
    assert np.abs(w - complexify(w_ref)).max() < 1e-11


@pytest.mark.parametrize("nspf,cluster", [(8, 1), (9, 1), (11, 1), (11, 0)],
                         ids=["2x1568", "4x2592", "cluster6050", "loop6050"])
def test_expoavecprop_long_vectors(built_lib, nspf, cluster):
    """4 electrons in 8, 9 and 11 orbitals: 784, 1296 and 3025 determinants, so the
    real-ified Krylov vectors have 1568 and 2592 entries (the register-resident
    Gram-Schmidt kernel with two and four values per thread) and 6050 (beyond 4096:
    the cluster kernel, one value per thread, or with kry_cluster = 0 the looping
    single-CTA kernel), against the oracle's DGEXPV."""
    from sincgpu import SincProject, WalkTables
    sysm = orc.SincSystem(15, 0.5, [[0, 0, 0]], [2.0])
    gpu = SincProject(15, 0.5, [[0, 0, 0]], [2.0], nspf)
    gpu.set_option("kry_cluster", cluster)
    try:
        gpu.ci_attach(WalkTables(4, nspf, 0))
        ow = CIWalks(4, nspf, 0)
        phi = orc.seeded_orbitals(sysm, nspf, seed=33)
        mat, _ = sysm.call_twoe_matel00(phi, phi)
        ph = np.conj(phi).T
        pot, ke, z = ph @ sysm.mult_pot(phi), ph @ sysm.mult_ke(phi), ph @ sysm.mult_zdipole(phi)
        gpu.assemble_sparsemats(mat, pot, ke, z)
        xp, xo, xk = ow.assemble_doubles(mat), ow.assemble_singles(pot), ow.assemble_singles(ke)
        rng = np.random.default_rng(34)
        a = rng.standard_normal(ow.numconfig) + 1j * rng.standard_normal(ow.numconfig)
        a /= np.linalg.norm(a)
        dt, m = 0.05, 12
        tf = -1j * dt
        mv = lambda x: realify(tf * ow.sparsesparsemult(complexify(x), xp, xo, xk,  # noqa: E731
                                                        constant=sysm.nucrepulsion))
        w_ref, g_ref, info = dgexpv(2 * ow.numconfig, m, 1.0, realify(a), 1e-9, dt, mv,
                                    lambda u, v: float(u @ v), 1.0, 2 * ow.numconfig - 1)
        w, g, nstep = gpu.expoavecprop(a, 1.0, krylovdim=m, tol=1e-9, anorm=dt, stepguess=1.0, timefac=tf)
        assert nstep == info["nstep"]
        assert g == pytest.approx(g_ref, rel=1e-12)
        assert np.abs(w - complexify(w_ref)).max() < 1e-11
    finally:
        gpu.close()


@pytest.mark.parametrize("nspf", [13, 14], ids=["cluster2x12168", "cluster4x16562"])
def test_expoavecprop_cluster_vs_one_cta(built_lib, nspf):
    """4 electrons in 13 and 14 orbitals (6084 and 8281 determinants: 12168 and 16562
    reals, the cluster Gram-Schmidt kernel with two and four values per thread)
    against the single-CTA kernel (kry_cluster = 0, checked against the oracle
    above): the same Krylov steps, the propagated vector to 1e-12 (the two differ
    in the shape of each dot product's sum only).  The Hamiltonian is the
    library's own on seeded orbitals."""
    from sincgpu import SincProject, WalkTables
    sysm = orc.SincSystem(13, 0.5, [[0, 0, 0]], [2.0])
    gpu = SincProject(13, 0.5, [[0, 0, 0]], [2.0], nspf)
    try:
        wt = WalkTables(4, nspf, 0)
        gpu.ci_attach(wt)
        phi = orc.seeded_orbitals(sysm, nspf, seed=35)
        mat, _ = gpu.call_twoe_matel00(phi)
        pot, ke, z = gpu.onebody_matel(phi)
        gpu.assemble_sparsemats(mat, pot, ke, z)
        rng = np.random.default_rng(36)
        a = rng.standard_normal(wt.numconfig) + 1j * rng.standard_normal(wt.numconfig)
        a /= np.linalg.norm(a)
        dt, m = 0.05, 12
        out = {}
        for cl in (0, 1):
            gpu.set_option("kry_cluster", cl)
            out[cl] = gpu.expoavecprop(a, 1.0, krylovdim=m, tol=1e-9, anorm=dt, stepguess=1.0, timefac=-1j * dt)
        assert out[0][2] == out[1][2]
        assert out[1][1] == pytest.approx(out[0][1], rel=1e-12)
        assert np.abs(out[1][0] - out[0][0]).max() < 1e-12
    finally:
        gpu.close()
