"""Precision form: Coulomb passes in FP32 (context option coulomb_fp32=1).

The pair products phi_a conj(phi_b) are formed in FP64 and rounded once; the
three forward and inverse FFT passes, twiddles and kernel spectrum are FP32;
the reduced potentials are widened to FP64 and every contraction after them
(twoematel, reducedpot, actreduced00, CI sigma) stays FP64.  Stated error
bounds against the FP64 oracle, relative to the largest magnitude:
  reduced potentials twoereduced   <= 1e-6
  twoematel                        <= 1e-6
  orbital RHS (actreduced00)       <= 1e-6
  CI energy <A|H|A>                <= 1e-6 (relative)
and the FP32 form must actually differ from FP64 (> 1e-10), which shows the
FP32 passes ran.
"""
import numpy as np
import pytest

from oracle import sinc_oracle as orc
from oracle.walks_oracle import CIWalks

pytestmark = pytest.mark.gpu
FP32_TOL = 1e-6
ENERGY_TOL = 1e-6


def relerr(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


@pytest.fixture(scope="module")
def sysgpu(built_lib):
    """Two Z=1 nuclei at z=+-1.2 (centershift -+4), 25^3 points, spacing 0.3, 6 orbitals."""
    from sincgpu import SincProject
    cs = [[0, 0, 4], [0, 0, -4]]
    sysm = orc.SincSystem(25, 0.3, cs, [1.0, 1.0])
    gpu = SincProject(25, 0.3, cs, [1.0, 1.0], 6)
    phi = orc.seeded_orbitals(sysm, 6, seed=51)
    mat_ref, red_ref = sysm.call_twoe_matel00(phi, phi)
    yield sysm, gpu, phi, mat_ref, red_ref
    gpu.set_option("coulomb_fp32", 0)
    gpu.close()


def test_fp32_twoe_matel_bounds(sysgpu):
    sysm, gpu, phi, mat_ref, red_ref = sysgpu
    gpu.set_option("coulomb_fp32", 1)
    try:
        mat, red = gpu.call_twoe_matel00(phi)
    finally:
        gpu.set_option("coulomb_fp32", 0)
    e_red, e_mat = relerr(red, red_ref), relerr(mat, mat_ref)
    print(f"fp32 twoereduced rel err {e_red:.2e}, twoematel rel err {e_mat:.2e}")
    assert 1e-10 < e_red < FP32_TOL
    assert 1e-10 < e_mat < FP32_TOL
    # Hermitian structure holds to the FP32 rounding level: mat(a,b,c,d) = conj(mat(b,a,d,c));
    # on the diagonal pairs (a,a) this is the FP32 imaginary residue of a real density's solve
    assert np.abs(mat - np.conj(mat.transpose(1, 0, 3, 2))).max() < 1e-7 * np.abs(mat).max()
    # back to FP64: plain-form bar again
    mat64, red64 = gpu.call_twoe_matel00(phi)
    assert relerr(red64, red_ref) < 1e-11
    assert relerr(mat64, mat_ref) < 1e-11


def test_fp32_op_tinv_bounds(sysgpu):
    sysm, gpu, _, _, _ = sysgpu
    rng = np.random.default_rng(52)
    dens = rng.standard_normal((sysm.G, 3)) + 1j * rng.standard_normal((sysm.G, 3))
    ref = sysm.op_tinv(dens)
    gpu.set_option("coulomb_fp32", 1)
    try:
        out = gpu.op_tinv(dens)
    finally:
        gpu.set_option("coulomb_fp32", 0)
    e = relerr(out, ref)
    print(f"fp32 op_tinv rel err {e:.2e}")
    assert 1e-10 < e < FP32_TOL


def test_fp32_orbital_rhs_bounds(sysgpu):
    sysm, gpu, phi, mat_ref, red_ref = sysgpu
    n = phi.shape[1]
    tally = orc.seeded_tally(n, seed=53)
    den = orc.seeded_hermitian_psd(n, seed=54)
    inv = orc.invmatsmooth(den)
    rp_ref = orc.get_reducedpot(red_ref, tally)
    out_ref = orc.actreduced00(sysm, phi, phi, den, inv, rp_ref)
    gpu.set_option("coulomb_fp32", 1)
    try:
        out, mat = gpu.orbital_rhs(phi, tally, den, inv)
    finally:
        gpu.set_option("coulomb_fp32", 0)
    e_rhs, e_mat = relerr(out, out_ref), relerr(mat, mat_ref)
    print(f"fp32 orbital RHS rel err {e_rhs:.2e}, twoematel {e_mat:.2e}")
    assert 1e-10 < e_rhs < FP32_TOL
    assert e_mat < FP32_TOL


def test_fp32_ci_energy_bound(sysgpu, built_lib):
    """<A|H|A> with H assembled from FP32-form twoematel vs the FP64 oracle."""
    from sincgpu import SincProject, WalkTables
    sysm, _, phi, mat_ref, _ = sysgpu
    n = phi.shape[1]
    cs = [[0, 0, 4], [0, 0, -4]]
    ow = CIWalks(2, n, 0)
    ph = np.conj(phi).T
    pot, ke, z = ph @ sysm.mult_pot(phi), ph @ sysm.mult_ke(phi), ph @ sysm.mult_zdipole(phi)
    rng = np.random.default_rng(55)
    a = rng.standard_normal(ow.numconfig) + 1j * rng.standard_normal(ow.numconfig)
    a /= np.linalg.norm(a)
    e_ref = np.vdot(a, ow.sparsesparsemult(a, ow.assemble_doubles(mat_ref), ow.assemble_singles(pot),
                                           ow.assemble_singles(ke), constant=sysm.nucrepulsion)).real
    with SincProject(25, 0.3, cs, [1.0, 1.0], n) as g:
        g.ci_attach(WalkTables(2, n, 0))
        g.set_option("coulomb_fp32", 1)
        mat, _ = g.call_twoe_matel00(phi)
        g.assemble_sparsemats(mat, pot, ke, z)
        e = np.vdot(a, g.sparseconfigmult(a)).real
    err = abs(e - e_ref) / abs(e_ref)
    print(f"fp32 CI energy {e:.12f} vs {e_ref:.12f}: rel err {err:.2e}")
    assert err < ENERGY_TOL


def test_option_validation(sysgpu):
    from sincgpu import SincGpuError
    gpu = sysgpu[1]
    with pytest.raises(SincGpuError):
        gpu.set_option("coulomb_fp32", 2)
    with pytest.raises(SincGpuError):
        gpu.set_option("no_such_option", 1)
