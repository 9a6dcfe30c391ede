"""The three-pass Coulomb form (option coul_fused = 1: x pass, then the y, z and
inverse-y transforms of each (pair, kx) plane in one kernel with the plane in
shared memory, split over a thread-block cluster where it does not fit one CTA,
then the inverse x pass) against the oracle and the five-pass form, through the
C ABI.  Covered: one CTA per plane (21^3, 25^3, 41^3 in FP64), clusters of 4
(81^3 in FP64) and 2 (81^3 in FP32).  Tolerances: 1e-11 against the oracle
(FP64), 1e-13 against the five-pass form (same transforms; the kernel spectrum
is taken real), the FP32 forms within 1e-6 of each other."""
import numpy as np
import pytest

from oracle import sinc_oracle as orc

pytestmark = pytest.mark.gpu


def relerr(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max())


@pytest.mark.parametrize("N,d,n", [(21, 0.4, 5), (25, 0.35, 4), (41, 0.25, 10)])
def test_pairs_match_oracle_and_five_pass(built_lib, N, d, n):
    from sincgpu import SincProject
    sysm = orc.SincSystem(N, d, [[0, 0, 0]], [2.0])
    gpu = SincProject(N, d, [[0, 0, 0]], [2.0], n)
    try:
        phi = orc.seeded_orbitals(sysm, n, seed=70 + N)
        gpu.set_option("coul_fused", 0)
        mat5, red5 = gpu.call_twoe_matel00(phi)
        gpu.set_option("coul_fused", 1)
        mat3, red3 = gpu.call_twoe_matel00(phi)
        mat_ref, red_ref = sysm.call_twoe_matel00(phi, phi, workers=4)
        assert relerr(red3, red_ref) < 1e-11
        assert relerr(mat3, mat_ref) < 1e-11
        assert relerr(red3, red5) < 1e-13
        assert relerr(mat3, mat5) < 1e-13
    finally:
        gpu.close()


def test_cluster_planes_81(built_lib):
    """81^3 (P = 162): the plane is split over clusters of 4 CTAs in FP64 and of 2
    in FP32; op_tinv on three densities."""
    from sincgpu import SincProject
    N, d = 81, 0.3
    cs = [[0, 0, 10], [0, 0, -10]]
    sysm = orc.SincSystem(N, d, cs, [3.0, 1.0])
    gpu = SincProject(N, d, cs, [3.0, 1.0], 2)
    try:
        assert gpu.fft_length == 162
        rng = np.random.default_rng(81)
        dens = rng.standard_normal((sysm.G, 3)) + 1j * rng.standard_normal((sysm.G, 3))
        gpu.set_option("coul_fused", 1)
        out3 = gpu.op_tinv(dens)
        assert relerr(out3, sysm.op_tinv(dens, workers=8)) < 1e-11
        gpu.set_option("coul_fused", 0)
        out5 = gpu.op_tinv(dens)
        assert relerr(out3, out5) < 1e-13
        gpu.set_option("coulomb_fp32", 1)
        f5 = gpu.op_tinv(dens)
        gpu.set_option("coul_fused", 1)
        f3 = gpu.op_tinv(dens)
        assert relerr(f3, f5) < 1e-6
        assert relerr(f3, out5) < 1e-5
    finally:
        gpu.close()


def test_orbital_rhs_avec_fused_workload_b(built_lib):
    """The benchmarked A-vector entry on the 41^3 / 10-orbital workload with the
    three-pass form equals the five-pass form to rounding."""
    from sincgpu import SincProject, WalkTables
    from sincgpu.inputs import WORKLOADS, seeded_avector, seeded_orbitals
    w = WORKLOADS["B"]
    gpu = SincProject(w.numpoints, w.spacing, w.centershift, w.nuccharges, w.nspf)
    try:
        wt = WalkTables(w.numelec, w.nspf, 0)
        gpu.ci_attach(wt)
        phi = seeded_orbitals(w.numpoints, w.spacing, w.nspf, seed=1)
        a = seeded_avector(wt.numconfig, seed=2)
        gpu.set_option("coul_fused", 0)
        o5 = gpu.orbital_rhs_avec(phi, a)
        gpu.set_option("coul_fused", 1)
        o3 = gpu.orbital_rhs_avec(phi, a)
        assert relerr(o3, o5) < 1e-13
    finally:
        gpu.close()


def test_paired_z_pass_162(built_lib):
    """The z pass with 9 threads per length-162 line (coul_z2 = 1: each thread one
    18-point and two 9-point sub-transforms) against the plain z pass (18 threads
    per line) and the oracle, FP64 and FP32."""
    from sincgpu import SincProject
    N, d = 81, 0.3
    sysm = orc.SincSystem(N, d, [[0, 0, 0]], [1.0])
    gpu = SincProject(N, d, [[0, 0, 0]], [1.0], 2)
    try:
        rng = np.random.default_rng(162)
        dens = rng.standard_normal((sysm.G, 2)) + 1j * rng.standard_normal((sysm.G, 2))
        for fp32 in (0, 1):
            gpu.set_option("coulomb_fp32", fp32)
            gpu.set_option("coul_z2", 0)
            plain = gpu.op_tinv(dens)
            gpu.set_option("coul_z2", 1)
            paired = gpu.op_tinv(dens)
            assert relerr(paired, plain) < 1e-14
            if not fp32:
                assert relerr(paired, sysm.op_tinv(dens, workers=8)) < 1e-11
        gpu.set_option("coul_z2", 0)
    finally:
        gpu.close()


def test_tma_z_pass_162(built_lib):
    """The TMA-staged z pass (coul_tma = 1) at length 162, where both it and the
    plain pass read the real spectrum over the whole table: agreement to 1e-14,
    the oracle to 1e-11, no timeouts (FP64 and FP32 against FP64)."""
    from sincgpu import SincProject
    N, d = 81, 0.3
    sysm = orc.SincSystem(N, d, [[0, 0, 0]], [1.0])
    gpu = SincProject(N, d, [[0, 0, 0]], [1.0], 2)
    try:
        rng = np.random.default_rng(164)
        dens = rng.standard_normal((sysm.G, 2)) + 1j * rng.standard_normal((sysm.G, 2))
        plain = gpu.op_tinv(dens)
        gpu.set_option("coul_tma", 1)
        staged = gpu.op_tinv(dens)
        assert relerr(staged, plain) < 1e-14
        assert relerr(staged, sysm.op_tinv(dens, workers=8)) < 1e-11
        gpu.set_option("coulomb_fp32", 1)
        assert relerr(gpu.op_tinv(dens), plain) < 1e-5
        assert gpu.kernel_timeouts() == [0, 0]
    finally:
        gpu.close()
