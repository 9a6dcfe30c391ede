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


@pytest.mark.parametrize("m,n,k", [(128, 16, 8), (300, 40, 37), (1000, 272, 272), (77, 256, 64), (129, 112, 110)])
def test_gemm_tf32x3_matches_fp64(proj, m, n, k):
    import torch
    g = torch.Generator().manual_seed(m * 7 + n * 3 + k)
    a = torch.randn(m, k, generator=g, dtype=torch.float64)
    b = torch.randn(n, k, generator=g, dtype=torch.float64)
    ref = (a @ b.T).numpy()
    da, db = a.cuda(), b.cuda()
    out = torch.full((m, n), float("nan"), dtype=torch.float64, device="cuda")
    assert proj.gemm_tf32x3_dev(da, db, out) == 0
    got = out.cpu().numpy()
    assert np.isfinite(got).all()
    err = np.abs(got - ref).max() / np.abs(ref).max()
    print(f"gemm_tf32x3 m={m} n={n} k={k}: max error / max |C| = {err:.3g}")
    assert err < 5e-6, err


def test_reducedpot_tf32_contraction(built_lib):
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
        p.orbital_rhs_avec_dev(phi, av, *bufs)
        p.set_option("contract_tf32", 0)
        red = bufs[4]
        err = (red - red64).abs().max().item() / red64.abs().max().item()
        rhs_err = (bufs[5] - out64).abs().max().item() / out64.abs().max().item()
        print(f"reducedpot 3xTF32: {err:.3g}, orbital RHS: {rhs_err:.3g}")
        assert err < 1e-6, err
        assert rhs_err < 1e-6, rhs_err
    finally:
        p.close()
