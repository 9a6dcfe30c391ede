"""GPU parity of the SINCDVR project drop-ins against the CPU oracle.

Every call goes through the C ABI (libsincgpu.so) via sincgpu.SincProject.
Tolerance: 1e-11 relative to the largest magnitude of the compared array
(the plain FP64 form's bar for reduced potentials and the orbital RHS).
"""
import numpy as np
import pytest

from oracle import sinc_oracle as orc

pytestmark = pytest.mark.gpu
TOL = 1e-11


def relerr(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.fixture(scope="module")
def he(built_lib):
    """Config A: He (Z=2 at the origin), 21^3 points, spacing 0.4, 5 orbitals."""
    from sincgpu import SincProject
    sysm = orc.SincSystem(21, 0.4, [[0, 0, 0]], [2.0])
    gpu = SincProject(21, 0.4, [[0, 0, 0]], [2.0], 5)
    phi = orc.seeded_orbitals(sysm, 5, seed=11)
    yield sysm, gpu, phi
    gpu.close()


@pytest.fixture(scope="module")
def h2(built_lib):
    """H2-like: two Z=1 nuclei at z=+-0.75 (centershift -+6), 41^3, spacing 0.25."""
    from sincgpu import SincProject
    cs = [[0, 0, 6], [0, 0, -6]]
    sysm = orc.SincSystem(41, 0.25, cs, [1.0, 1.0])
    gpu = SincProject(41, 0.25, cs, [1.0, 1.0], 10)
    yield sysm, gpu
    gpu.close()


def test_tables_match_oracle(he, h2):
    for sysm, gpu in ((he[0], he[1]), h2):
        t = gpu.get_tables()
        assert relerr(t["tempcoulomb"], sysm.tempcoulomb) < 1e-12
        assert relerr(t["pot"], sysm.pot) < 1e-12
        assert relerr(t["kevect"], sysm.kevect) < 1e-15
        assert abs(t["nucrepulsion"] - sysm.nucrepulsion) < 1e-14


def test_fft_length_is_smooth(he, h2):
    assert he[1].fft_length == 42   # 2*21-1 = 41 -> 42 = 2*3*7
    assert h2[1].fft_length == 81   # 2*41-1 = 81 = 3^4


def test_op_tinv(he):
    sysm, gpu, _ = he
    rng = np.random.default_rng(3)
    dens = rng.standard_normal((sysm.G, 3)) + 1j * rng.standard_normal((sysm.G, 3))
    ref = sysm.op_tinv(dens)
    out = gpu.op_tinv(dens, circsize=1)
    assert relerr(out, ref) < TOL


def test_op_tinv_h2_subset(h2):
    sysm, gpu = h2
    rng = np.random.default_rng(4)
    dens = rng.standard_normal((sysm.G, 2)) + 1j * rng.standard_normal((sysm.G, 2))
    assert relerr(gpu.op_tinv(dens), sysm.op_tinv(dens)) < TOL


def test_call_twoe_matel00_hermitian(he):
    sysm, gpu, phi = he
    mat_ref, red_ref = sysm.call_twoe_matel00(phi, phi)
    mat, red = gpu.call_twoe_matel00(phi)
    assert relerr(red, red_ref) < TOL
    assert relerr(mat, mat_ref) < TOL


def test_call_twoe_matel00_general(he):
    sysm, gpu, phi = he
    phi2 = orc.seeded_orbitals(sysm, 5, seed=12)
    mat_ref, red_ref = sysm.call_twoe_matel00(phi, phi2)
    mat, red = gpu.call_twoe_matel00(phi, phi2)
    assert relerr(red, red_ref) < TOL
    assert relerr(mat, mat_ref) < TOL


@pytest.mark.parametrize("nspf,general,symdiag", [(12, False, 0), (12, False, 1), (16, False, 1), (9, True, 1)])
def test_call_twoe_matel00_multitile(built_lib, nspf, general, symdiag):
    """Pair lists longer than one GEMM tile (2U = 156 and 272 hermitian, 2n^2 = 162
    general): only the upper-triangle tiles of the symmetric pair matrix are
    computed and the lower ones mirrored; with twoe_symdiag the diagonal tiles
    compute their lower 8 x 8 blocks only (hermitian pairs)."""
    from sincgpu import SincProject
    sysm = orc.SincSystem(21, 0.4, [[0, 0, 0]], [2.0])
    gpu = SincProject(21, 0.4, [[0, 0, 0]], [2.0], nspf)
    gpu.set_option("twoe_symdiag", symdiag)
    try:
        phi = orc.seeded_orbitals(sysm, nspf, seed=21)
        phi2 = orc.seeded_orbitals(sysm, nspf, seed=22) if general else phi
        mat_ref, red_ref = sysm.call_twoe_matel00(phi, phi2)
        mat, red = gpu.call_twoe_matel00(phi, phi2) if general else gpu.call_twoe_matel00(phi)
        assert relerr(red, red_ref) < TOL
        assert relerr(mat, mat_ref) < TOL
    finally:
        gpu.close()


def test_coulomb_tma_z_pass_matches_plain(h2):
    """The TMA-staged persistent z pass (option coul_tma = 1; the automatic choice
    is the plain pass) against the plain z pass on the same densities: same transforms, the kernel spectrum's real part only (its
    imaginary part is rounding noise), so agreement to 1e-14; no timeouts."""
    sysm, gpu = h2
    rng = np.random.default_rng(7)
    dens = rng.standard_normal((sysm.G, 3)) + 1j * rng.standard_normal((sysm.G, 3))
    gpu.set_option("coul_tma", 0)
    plain = gpu.op_tinv(dens)
    gpu.set_option("coul_tma", 1)
    staged = gpu.op_tinv(dens)
    assert relerr(staged, plain) < 1e-14
    assert relerr(staged, sysm.op_tinv(dens)) < TOL
    assert gpu.kernel_timeouts() == [0, 0]


def test_pair_chunking_is_exact(h2):
    """Each pair's Coulomb solve is independent of the others, so the pair-chunk
    size (automatic: the whole list within a 2 GB budget) changes nothing: chunks
    of 3 pairs give bitwise the same reduced potentials and twoematel."""
    sysm, gpu = h2
    phi = orc.seeded_orbitals(sysm, 10, seed=31)
    mat0, red0 = gpu.call_twoe_matel00(phi)
    gpu.set_option("coul_chunk", 3)
    try:
        mat3, red3 = gpu.call_twoe_matel00(phi)
    finally:
        gpu.set_option("coul_chunk", 0)
    assert np.array_equal(red0, red3)
    assert np.array_equal(mat0, mat3)


def test_mult_ke(he, h2):
    for sysm, gpu in ((he[0], he[1]), h2):
        rng = np.random.default_rng(5)
        x = rng.standard_normal((sysm.G, 3)) + 1j * rng.standard_normal((sysm.G, 3))
        assert relerr(gpu.mult_ke(x), sysm.mult_ke(x)) < TOL


def test_get_and_mult_reducedpot(he):
    sysm, gpu, phi = he
    _, red = sysm.call_twoe_matel00(phi, phi)
    tally = orc.seeded_tally(5, seed=6)
    rp_ref = orc.get_reducedpot(red, tally)
    rp = gpu.get_reducedpot(red, tally)
    assert relerr(rp, rp_ref) < TOL
    out_ref = orc.mult_reducedpot(phi, rp_ref)
    assert relerr(gpu.mult_reducedpot(phi, rp_ref), out_ref) < TOL
    # window of orbitals (firstspf:lastspf)
    out = gpu.mult_reducedpot(phi, rp_ref[:, :, 1:4], firstspf=2, lastspf=4)
    assert relerr(out, out_ref[:, 1:4]) < TOL


@pytest.mark.parametrize("dentimeflag,projflag,ztd", [(1, 1, 0.0), (1, 1, 0.05), (0, 0, 0.0), (1, 0, 0.0)])
def test_actreduced00(he, dentimeflag, projflag, ztd):
    sysm, gpu, phi = he
    _, red = sysm.call_twoe_matel00(phi, phi)
    tally = orc.seeded_tally(5, seed=7)
    rp = orc.get_reducedpot(red, tally)
    den = orc.seeded_hermitian_psd(5, seed=8)
    inv = orc.invmatsmooth(den)
    ref = orc.actreduced00(sysm, phi, phi, den, inv, rp, dentimeflag=dentimeflag, projflag=projflag,
                           ztdpot=ztd)
    out = gpu.actreduced00(phi, phi, den, inv, rp, dentimeflag=dentimeflag, projflag=projflag, ztdpot=ztd)
    assert relerr(out, ref) < TOL


def test_from_tables_matches(he, built_lib):
    from sincgpu import SincProject
    sysm, gpu, phi = he
    g2 = SincProject.from_tables(21, 0.4, 5, sysm.threed_two.astype(np.complex128), sysm.pot)
    try:
        m1, r1 = gpu.call_twoe_matel00(phi)
        m2, r2 = g2.call_twoe_matel00(phi)
        assert relerr(r2, r1) < 1e-12
        assert relerr(g2.mult_ke(phi), gpu.mult_ke(phi)) < 1e-14
    finally:
        g2.close()


def test_even_grid_odd_shift(built_lib):
    """Even N requires odd centershift (sincproject.f90:196-204)."""
    from sincgpu import SincProject, SincGpuError
    sysm = orc.SincSystem(12, 0.5, [[1, -1, 3]], [1.0])
    gpu = SincProject(12, 0.5, [[1, -1, 3]], [1.0], 3)
    try:
        t = gpu.get_tables()
        assert relerr(t["pot"], sysm.pot) < 1e-12
        phi = orc.seeded_orbitals(sysm, 3, seed=2)
        m, r = gpu.call_twoe_matel00(phi)
        mr, rr = sysm.call_twoe_matel00(phi, phi)
        assert relerr(r, rr) < TOL and relerr(m, mr) < TOL
    finally:
        gpu.close()
    with pytest.raises(SincGpuError):
        SincProject(12, 0.5, [[0, 0, 0]], [1.0], 3)
