"""Orbital propagation (expospfprop -> DGPHIV, jacoperate, spf_orthogit) on the
GPU against the oracle's restatement of the same algorithm.

Tolerances: orthonormalisation 1e-12, propagated orbitals 1e-10 relative to
max|phi| (FP64; Krylov vectors and the Pade exponential reorder sums relative to
the oracle); Krylov step counts, Jacobian-product counts and the saved
dimension / step-size state must agree exactly.
"""
import numpy as np
import pytest

from oracle import orbprop_oracle as op
from oracle import sinc_oracle as orc

pytestmark = pytest.mark.gpu


def dev(torch, a):
    """Fortran-ordered numpy array -> CUDA tensor with the same memory layout."""
    return torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=np.complex128).T)).cuda()


def host(t):
    return t.cpu().numpy().T


@pytest.fixture(scope="module")
def system(built_lib):
    import torch
    from sincgpu import SincProject
    n = 4
    sysm = orc.SincSystem(13, 0.5, [[0, 0, 0]], [2.0], toothnbig=40, toothnsmall=10)
    gpu = SincProject(13, 0.5, [[0, 0, 0]], [2.0], n, toothnbig=40, toothnsmall=10)
    phi = orc.seeded_orbitals(sysm, n, seed=71)
    _, red = sysm.call_twoe_matel00(phi, phi)
    slots = []
    for s in range(2):
        den = orc.seeded_hermitian_psd(n, seed=72 + s)
        slots.append((den, orc.invmatsmooth(den), orc.get_reducedpot(red, orc.seeded_tally(n, seed=74 + s))))
    dslots = [tuple(dev(torch, x) for x in sl) for sl in slots]
    yield sysm, gpu, phi, slots, dslots
    gpu.close()


def test_spf_orthogit(system):
    import torch
    sysm, gpu, phi, _, _ = system
    rng = np.random.default_rng(76)
    bad = phi + 0.05 * (rng.standard_normal(phi.shape) + 1j * rng.standard_normal(phi.shape)) * np.abs(phi)
    ref, err_ref = op.spf_orthogit(bad)
    d = dev(torch, bad)
    err = gpu.spf_orthogit_dev(d)
    out = host(d)
    assert np.abs(out - ref).max() < 1e-12
    assert np.abs(np.conj(out).T @ out - np.eye(phi.shape[1])).max() < 1e-13
    assert err == pytest.approx(err_ref, abs=1e-14)


@pytest.mark.parametrize("linear", [True, False], ids=["linear", "slot0"])
def test_expospfprop_matches_oracle(system, linear):
    import torch
    sysm, gpu, phi, slots, dslots = system
    dt = 0.05
    st = op.OrbPropState(expodim=8, maxexpodim=30, expostepfac=1.2, first_stepsize=dt)
    gpu.orbprop_setup(8, 30, 1.2, dt)
    ref, info = op.expospfprop(sysm, st, phi, slots, 0.0, dt, 0.0, dt, linear, expotol=1e-8)
    d = dev(torch, phi)
    iters = gpu.expospfprop_dev(d, dslots[0], dslots[1] if linear else None, 0.0, dt, 0.0, dt, linear,
                                expotol=1e-8)
    out = host(d)
    assert iters == info["numiters"]
    s = gpu.orbprop_state()
    assert (s["thisexpodim"], s["exposet"], s["icalled"]) == (st.thisexpodim, st.exposet, st.icalled)
    assert s["tempstepsize"] == pytest.approx(st.tempstepsize, rel=1e-12)
    assert np.abs(out - ref).max() < 1e-10 * np.abs(ref).max()
    assert np.abs(np.conj(out).T @ out - np.eye(phi.shape[1])).max() < 1e-13


def test_expospfprop_state_over_calls(system):
    """Consecutive calls with a small first step force several internal Krylov
    steps, growth of the dimension and the step guess hand-over."""
    import torch
    sysm, gpu, phi, slots, dslots = system
    st = op.OrbPropState(expodim=5, maxexpodim=12, expostepfac=1.2, first_stepsize=0.002)
    gpu.orbprop_setup(5, 12, 1.2, 0.002)
    ref = phi.copy()
    d = dev(torch, phi)
    t = 0.0
    for k in range(3):
        dt = 0.08
        ref, info = op.expospfprop(sysm, st, ref, slots, t, t + dt, t, t + dt, True, expotol=1e-9)
        iters = gpu.expospfprop_dev(d, dslots[0], dslots[1], t, t + dt, t, t + dt, True, expotol=1e-9)
        s = gpu.orbprop_state()
        assert iters == info["numiters"], k
        assert (s["thisexpodim"], s["exposet"], s["icalled"]) == (st.thisexpodim, st.exposet, st.icalled), k
        assert s["tempstepsize"] == pytest.approx(st.tempstepsize, rel=1e-12), k
        t += dt
    out = host(d)
    assert np.abs(out - ref).max() < 1e-10 * np.abs(ref).max()


def test_orthogonalisation_fused_is_bitwise(system):
    """The one-launch Arnoldi orthogonalisation (bounded grid barriers) gives the
    same bits, step counts and saved state as the dot / projection / norm launches."""
    import torch
    sysm, gpu, phi, slots, dslots = system
    outs = []
    try:
        for fused in (1, 0):
            gpu.set_option("orth_fused", fused)
            gpu.orbprop_setup(5, 12, 1.2, 0.002)
            d = dev(torch, phi)
            iters = [gpu.expospfprop_dev(d, dslots[0], dslots[1], t, t + 0.08, t, t + 0.08, True, expotol=1e-9)
                     for t in (0.0, 0.08)]
            outs.append((host(d), iters, gpu.orbprop_state()))
    finally:
        gpu.set_option("orth_fused", 1)
    assert np.array_equal(outs[0][0], outs[1][0])
    assert outs[0][1] == outs[1][1] and outs[0][2] == outs[1][2]


def test_blended_potential_matches_per_slot(system):
    """The Jacobian reading one blended reduced potential Q and matrix M, formed
    once per call (orb_blendq = 1, the default), against the per-slot blend
    (orb_blendq = 0): the same Krylov steps and saved state, the propagated
    orbitals to 1e-12 (the same algebra, summed in another order)."""
    import torch
    sysm, gpu, phi, slots, dslots = system
    outs = []
    try:
        for bq in (1, 0):
            gpu.set_option("orb_blendq", bq)
            gpu.orbprop_setup(5, 12, 1.2, 0.002)
            d = dev(torch, phi)
            iters = [gpu.expospfprop_dev(d, dslots[0], dslots[1], t, t + 0.08, t, t + 0.08, True, expotol=1e-9)
                     for t in (0.0, 0.08)]
            outs.append((host(d), iters, gpu.orbprop_state()))
    finally:
        gpu.set_option("orb_blendq", 1)
    assert outs[0][1] == outs[1][1]
    assert outs[0][2]["thisexpodim"] == outs[1][2]["thisexpodim"]
    assert np.abs(outs[0][0] - outs[1][0]).max() < 1e-12 * np.abs(outs[1][0]).max()


def test_expospfprop_rejects_bad_setup(system):
    from sincgpu import SincGpuError
    gpu = system[1]
    with pytest.raises(SincGpuError):
        gpu.orbprop_setup(10, 200, 1.2, 0.05)
    with pytest.raises(SincGpuError):
        gpu.orbprop_setup(10, 100, 1.2, -1.0)
