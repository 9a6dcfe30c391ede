"""GPU parity of the fused orbital-RHS entries against the oracle.

sincgpu_orbital_rhs: (phi, tally, denmat, invdenmat) -> actreduced00 output and
twoematel in one call (the chain call_twoe_matel00 -> get_reducedpot ->
actreduced00 of SINCDVR/coreproject.f90 and MCTDH.SRC/mean.f90).
sincgpu_orbital_rhs_avec: (phi, A-vector) -> the same, with the 1-RDM, its
regularised inverse and the 2-RDM tally computed from the A-vector on the GPU
(getdenmat00 / get_tworeducedx of MCTDH.SRC).  Tolerance 1e-11 relative
(FP64 plain form).
"""
import numpy as np
import pytest

from oracle import sinc_oracle as orc
from oracle.walks_oracle import CIWalks

pytestmark = pytest.mark.gpu
TOL = 1e-11


def relerr(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


@pytest.fixture(scope="module")
def li(built_lib):
    """Z=3 at the origin, 19^3 points, spacing 0.45, 6 orbitals, 3 electrons (ms=1)."""
    from sincgpu import SincProject, WalkTables
    n = 6
    sysm = orc.SincSystem(19, 0.45, [[0, 0, 0]], [3.0])
    gpu = SincProject(19, 0.45, [[0, 0, 0]], [3.0], n)
    gpu.ci_attach(WalkTables(3, n, 1))
    ow = CIWalks(3, n, 1)
    phi = orc.seeded_orbitals(sysm, n, seed=41)
    rng = np.random.default_rng(42)
    a = rng.standard_normal(ow.numconfig) + 1j * rng.standard_normal(ow.numconfig)
    a /= np.linalg.norm(a)
    yield sysm, gpu, ow, phi, a
    gpu.close()


@pytest.mark.parametrize("timefac,ztd", [(-1j, 0.0), (-1j, 0.03), (-1.0, 0.0)])
def test_orbital_rhs(li, timefac, ztd):
    sysm, gpu, _, phi, _ = li
    n = phi.shape[1]
    tally = orc.seeded_tally(n, seed=43)
    den = orc.seeded_hermitian_psd(n, seed=44)
    inv = orc.invmatsmooth(den)
    mat_ref, red_ref = sysm.call_twoe_matel00(phi, phi)
    rp_ref = orc.get_reducedpot(red_ref, tally)
    out_ref = orc.actreduced00(sysm, phi, phi, den, inv, rp_ref, timefac=timefac, ztdpot=ztd)
    out, mat = gpu.orbital_rhs(phi, tally, den, inv, timefac=timefac, ztdpot=ztd)
    assert relerr(mat, mat_ref) < TOL
    assert relerr(out, out_ref) < TOL


@pytest.mark.parametrize("ztd", [0.0, 0.02])
def test_orbital_rhs_avec(li, ztd):
    sysm, gpu, ow, phi, a = li
    den = ow.getdenmat00(a)
    inv = orc.invmatsmooth(den)
    tally = ow.get_tworeducedx(a)
    _, red = sysm.call_twoe_matel00(phi, phi)
    rp = orc.get_reducedpot(red, tally)
    ref = orc.actreduced00(sysm, phi, phi, den, inv, rp, ztdpot=ztd)
    out = gpu.orbital_rhs_avec(phi, a, ztdpot=ztd)
    assert relerr(out, ref) < TOL


def test_orbital_rhs_avec_repeatable(li):
    """Deterministic reductions: two evaluations are bitwise equal."""
    _, gpu, _, phi, a = li
    o1 = gpu.orbital_rhs_avec(phi, a)
    o2 = gpu.orbital_rhs_avec(phi, a)
    assert np.array_equal(o1, o2)


def test_orbital_rhs_avec_overlap_is_bitwise(li):
    """The CI part and the kinetic contraction on the side stream (rhs_overlap = 1,
    the default) change only when work runs, not what it computes."""
    _, gpu, _, phi, a = li
    o1 = gpu.orbital_rhs_avec(phi, a, ztdpot=0.02)
    gpu.set_option("rhs_overlap", 0)
    try:
        o0 = gpu.orbital_rhs_avec(phi, a, ztdpot=0.02)
    finally:
        gpu.set_option("rhs_overlap", 1)
    assert np.array_equal(o0, o1)


def test_scheduling_options_reject_bad_values(li):
    from sincgpu import SincGpuError
    gpu = li[1]
    for name, bad in (("rhs_overlap", 2), ("orth_fused", -1), ("twoe_tile", 1), ("twoe_tile", 10),
                      ("rhs_upload_groups", 0), ("rhs_upload_groups", 9)):
        with pytest.raises(SincGpuError):
            gpu.set_option(name, bad)
    gpu.set_option("rhs_overlap", 1)
    gpu.set_option("orth_fused", 1)
    gpu.set_option("twoe_tile", 0)


def test_avec_reducedpot_mirror_equals_full(li):
    """The A-vector entry computes only the k <= i half of reducedpot and mirrors
    it (its 2-RDM comes from one A-vector); it equals the full product of the
    general mean-field entry on the same 2-RDM to rounding."""
    import torch
    sysm, gpu, ow, phi, a = li
    n, G = phi.shape[1], sysm.G
    cx = dict(dtype=torch.complex128, device="cuda")
    dphi = torch.from_numpy(np.ascontiguousarray(phi.T)).cuda()
    da = torch.from_numpy(a).cuda()
    den, inv = torch.empty((n, n), **cx), torch.empty((n, n), **cx)
    tally, mat = torch.empty((n,) * 4, **cx), torch.empty((n,) * 4, **cx)
    rp_half, rp_full, out = torch.empty((n, n, G), **cx), torch.empty((n, n, G), **cx), torch.empty((n, G), **cx)
    gpu.orbital_rhs_avec_dev(dphi, da, den, inv, tally, mat, rp_half, out)
    gpu.mean_field_dev(dphi, tally, mat, rp_full)
    torch.cuda.synchronize()
    err = float((rp_half - rp_full).abs().max() / rp_full.abs().max())
    assert err < 1e-13


@pytest.mark.parametrize("n", [7, 10])
def test_reducedpot_dmma_matches_dfma(built_lib, n):
    """The FP64 tensor-core (DMMA) reducedpot and twoematel GEMMs against the
    register-tiled DFMA ones on the same mean-field inputs: both FP64, different
    summation order.  n = 10 runs the widest one-tile instances (twoematel tile
    R = 7, reducedpot FN = 7 with the fused apply)."""
    import torch
    from oracle import sinc_oracle as orc
    from sincgpu import SincProject, WalkTables
    p = SincProject(21, 0.4, [[0, 0, 0]], [2.0], n)
    try:
        sysm = orc.SincSystem(21, 0.4, [[0, 0, 0]], [2.0])
        phi = torch.from_numpy(np.ascontiguousarray(orc.seeded_orbitals(sysm, n, seed=9).T)).cuda()
        w = WalkTables(2, n, 0)
        p.ci_attach(w)
        rng = np.random.default_rng(10)
        av = rng.standard_normal(w.numconfig) + 1j * rng.standard_normal(w.numconfig)
        av = torch.from_numpy(av / np.linalg.norm(av)).cuda()
        cx = dict(dtype=torch.complex128, device="cuda")
        bufs = [torch.empty((n, n), **cx), torch.empty((n, n), **cx), torch.empty((n,) * 4, **cx),
                torch.empty((n,) * 4, **cx), torch.empty((n, n, sysm.G), **cx), torch.empty((n, sysm.G), **cx)]
        p.set_option("rp_dmma", 0)
        p.set_option("twoe_dmma", 0)
        p.orbital_rhs_avec_dev(phi, av, *bufs)
        ref, ref_mat = bufs[4].clone(), bufs[3].clone()
        p.set_option("rp_dmma", 1)
        p.set_option("twoe_dmma", 1)
        p.orbital_rhs_avec_dev(phi, av, *bufs)
        err = (bufs[4] - ref).abs().max().item() / ref.abs().max().item()
        assert err < 1e-13, err
        err = (bufs[3] - ref_mat).abs().max().item() / ref_mat.abs().max().item()
        assert err < 1e-13, err
    finally:
        p.close()


@pytest.mark.parametrize("n,numelec,ms", [(8, 3, 1), (9, 2, 0), (10, 2, 0)])
def test_orbital_rhs_avec_wide_column_tiles(built_lib, n, numelec, ms):
    """The A-vector entry at 8, 9 and 10 orbitals: n(n+1) = 72, 90, 110 half
    columns, so the fused reducedpot + apply kernel runs its FN = 5, 6, 7
    instances and twoematel its R = 5, 6, 7 one-tile symmetric instances (the
    instances behind the 41^3 / 10-orbital benchmark), against the oracle."""
    from sincgpu import SincProject, WalkTables
    sysm = orc.SincSystem(15, 0.5, [[0, 0, 2], [0, 0, -2]], [1.0, 2.0])
    gpu = SincProject(15, 0.5, [[0, 0, 2], [0, 0, -2]], [1.0, 2.0], n)
    try:
        gpu.ci_attach(WalkTables(numelec, n, ms))
        ow = CIWalks(numelec, n, ms)
        phi = orc.seeded_orbitals(sysm, n, seed=50 + n)
        rng = np.random.default_rng(60 + n)
        a = rng.standard_normal(ow.numconfig) + 1j * rng.standard_normal(ow.numconfig)
        a /= np.linalg.norm(a)
        den = ow.getdenmat00(a)
        inv = orc.invmatsmooth(den)
        tally = ow.get_tworeducedx(a)
        _, red = sysm.call_twoe_matel00(phi, phi)
        rp = orc.get_reducedpot(red, tally)
        ref = orc.actreduced00(sysm, phi, phi, den, inv, rp, ztdpot=0.01)
        out = gpu.orbital_rhs_avec(phi, a, ztdpot=0.01)
        assert relerr(out, ref) < TOL
    finally:
        gpu.close()
