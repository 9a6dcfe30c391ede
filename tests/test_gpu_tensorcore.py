"""Tensor-core (tcgen05 kind::tf32, 3xTF32) contraction of the precision form,
through the C ABI: the raw GEMM against an FP64 product, and reducedpot with the
contraction option on against the FP64 path.

Tolerances: 3xTF32 keeps about 21 bits per product, and the tensor core adds the
products of each K = 8 step into the FP32 accumulator, so the error grows with K
(2.9e-6 of the largest |C| measured at K = 272 on random normal operands); the GEMM
is checked at 5e-6 of the largest |C| (plain TF32 would be ~1e-3, a wrong operand
layout O(1)); reducedpot and the orbital RHS at 1e-6 of their largest magnitude,
the precision form's orbital-RHS budget."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def proj(built_lib):
    from sincgpu import SincProject
    p = SincProject(21, 0.4, [[0, 0, 0]], [2.0], 5)
    yield p
    p.close()


MODES = {"kc16": {"tc_kc": 16, "tc_pipe": 0}, "kc32": {"tc_kc": 32, "tc_pipe": 0},
         "ring": {"tc_kc": 16, "tc_pipe": 1}, "ring4": {"tc_kc": 16, "tc_pipe": 2},
         "ring8": {"tc_kc": 16, "tc_pipe": 3}, "bulk": {"tc_kc": 16, "tc_pipe": 4},
         "bulk5": {"tc_kc": 16, "tc_pipe": 5}}


def set_mode(p, mode):
    for name, v in MODES[mode].items():
        p.set_option(name, v)


@pytest.mark.parametrize("mode", list(MODES))
@pytest.mark.parametrize("m,n,k", [(128, 16, 8), (300, 40, 37), (1000, 272, 272), (77, 256, 64), (129, 112, 110)])
def test_gemm_tf32x3_matches_fp64(proj, m, n, k, mode):
    """The three forms of the kernel: K chunks of 16 (two CTAs per SM), of 32, and
    the ring of staged chunks with a separate MMA-issuing warp (tc_pipe)."""
    import torch
    g = torch.Generator().manual_seed(m * 7 + n * 3 + k)
    a = torch.randn(m, k, generator=g, dtype=torch.float64)
    b = torch.randn(n, k, generator=g, dtype=torch.float64)
    ref = (a @ b.T).numpy()
    da, db = a.cuda(), b.cuda()
    out = torch.full((m, n), float("nan"), dtype=torch.float64, device="cuda")
    set_mode(proj, mode)
    try:
        assert proj.gemm_tf32x3_dev(da, db, out) == 0
    finally:
        set_mode(proj, "bulk")
    assert proj.kernel_timeouts()[0] == 0
    got = out.cpu().numpy()
    assert np.isfinite(got).all()
    err = np.abs(got - ref).max() / np.abs(ref).max()
    print(f"gemm_tf32x3 m={m} n={n} k={k}: max error / max |C| = {err:.3g}")
    assert err < 5e-6, err


@pytest.mark.parametrize("mode", ["kc16", "ring", "bulk"])
def test_reducedpot_tf32_contraction(built_lib, mode):
    import torch
    from oracle import sinc_oracle as orc
    from sincgpu import SincProject, WalkTables
    n = 6
    p = SincProject(21, 0.4, [[0, 0, 0]], [2.0], n)
    try:
        sysm = orc.SincSystem(21, 0.4, [[0, 0, 0]], [2.0])
        phi = torch.from_numpy(np.ascontiguousarray(orc.seeded_orbitals(sysm, n, seed=5).T)).cuda()
        w = WalkTables(2, n, 0)
        p.ci_attach(w)
        rng = np.random.default_rng(6)
        av = rng.standard_normal(w.numconfig) + 1j * rng.standard_normal(w.numconfig)
        av = torch.from_numpy(av / np.linalg.norm(av)).cuda()
        cx = dict(dtype=torch.complex128, device="cuda")
        G = sysm.G
        bufs = [torch.empty((n, n), **cx), torch.empty((n, n), **cx), torch.empty((n,) * 4, **cx),
                torch.empty((n,) * 4, **cx), torch.empty((n, n, G), **cx), torch.empty((n, G), **cx)]
        p.orbital_rhs_avec_dev(phi, av, *bufs)
        red64 = bufs[4].clone()
        out64 = bufs[5].clone()
        p.set_option("contract_tf32", 1)
        set_mode(p, mode)
        p.orbital_rhs_avec_dev(phi, av, *bufs)
        p.set_option("contract_tf32", 0)
        assert p.kernel_timeouts()[0] == 0
        red = bufs[4]
        err = (red - red64).abs().max().item() / red64.abs().max().item()
        rhs_err = (bufs[5] - out64).abs().max().item() / out64.abs().max().item()
        print(f"reducedpot 3xTF32: {err:.3g}, orbital RHS: {rhs_err:.3g}")
        assert err < 1e-6, err
        assert rhs_err < 1e-6, rhs_err
    finally:
        p.close()


@pytest.mark.parametrize("N,d,howmany", [(21, 0.4, 3), (41, 0.25, 2)])
def test_kinetic_tf32_contraction(built_lib, N, d, howmany):
    """The kinetic contraction on the tcgen05 tensor cores (option ke_tf32: one
    3xTF32 GEMM per axis, the lines of the grid against the N x N sine-DVR matrix)
    against the FP64 tensor-core path and the oracle, within 1e-6 of the largest
    magnitude; and the orbital RHS with it."""
    import torch
    from oracle import sinc_oracle as orc
    from sincgpu import SincProject
    p = SincProject(N, d, [[0, 0, 0]], [2.0], howmany)
    try:
        sysm = orc.SincSystem(N, d, [[0, 0, 0]], [2.0])
        phi = orc.seeded_orbitals(sysm, howmany, seed=N)
        ref = sysm.mult_ke(phi)
        dphi = torch.from_numpy(np.ascontiguousarray(phi.T)).cuda()
        out64 = torch.empty_like(dphi)
        out32 = torch.full_like(dphi, float("nan"))
        p.mult_ke_dev(dphi, out64, howmany)
        p.set_option("ke_tf32", 1)
        p.mult_ke_dev(dphi, out32, howmany)
        p.set_option("ke_tf32", 0)
        torch.cuda.synchronize()
        a64, a32 = out64.cpu().numpy().T, out32.cpu().numpy().T
        assert np.isfinite(a32).all()
        assert np.abs(a64 - ref).max() / np.abs(ref).max() < 1e-11
        err = np.abs(a32 - ref).max() / np.abs(ref).max()
        print(f"kinetic 3xTF32 N={N}: {err:.3g}")
        assert err < 1e-6, err
    finally:
        p.close()


def test_orbital_rhs_with_kinetic_tf32(built_lib):
    """The orbital RHS (the potential and z-field terms ride in the first axis's
    epilogue) with ke_tf32 and contract_tf32 against the FP64 form at 1e-6."""
    from oracle import sinc_oracle as orc
    from sincgpu import SincProject, WalkTables
    n = 5
    p = SincProject(21, 0.4, [[0, 0, 0]], [2.0], n)
    try:
        sysm = orc.SincSystem(21, 0.4, [[0, 0, 0]], [2.0])
        phi = orc.seeded_orbitals(sysm, n, seed=8)
        w = WalkTables(2, n, 0)
        p.ci_attach(w)
        rng = np.random.default_rng(9)
        av = rng.standard_normal(w.numconfig) + 1j * rng.standard_normal(w.numconfig)
        av /= np.linalg.norm(av)
        o64 = p.orbital_rhs_avec(phi, av, ztdpot=0.02)
        p.set_option("ke_tf32", 1)
        p.set_option("contract_tf32", 1)
        o32 = p.orbital_rhs_avec(phi, av, ztdpot=0.02)
        err = np.abs(o32 - o64).max() / np.abs(o64).max()
        print(f"orbital RHS, kinetic + reducedpot 3xTF32: {err:.3g}")
        assert err < 1e-6, err
    finally:
        p.close()
