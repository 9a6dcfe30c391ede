"""Constant-mean-field propagation step (cmf_prop_wfn with prepropflag=1,
step_flag=2, postpropflag=2) on the GPU against the oracle's restatement.

Every call goes through the C ABI.  Tolerances: energies 1e-10 relative, the
propagated orbitals and A-vector 1e-9 relative to their largest magnitude
(two Krylov propagators, four A-vector propagations and two mean-field builds
per step reorder FP64 sums relative to the oracle); Krylov products counts
must agree exactly.
"""
import numpy as np
import pytest

from oracle import sinc_oracle as orc
from oracle.cmf_oracle import CmfOracle, CmfParams, Pulse, pulse_ez
from oracle.walks_oracle import CIWalks

pytestmark = pytest.mark.gpu


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=np.complex128).T)).cuda()


def host(t):
    return t.cpu().numpy().T


@pytest.fixture(scope="module")
def base(built_lib):
    n = 4
    sysm = orc.SincSystem(11, 0.5, [[0, 0, 0]], [2.0], toothnbig=40, toothnsmall=10)
    phi = orc.seeded_orbitals(sysm, n, seed=91)
    nc = CIWalks(2, n, 0).numconfig
    rng = np.random.default_rng(92)
    a = rng.standard_normal(nc) + 1j * rng.standard_normal(nc)
    return sysm, phi, a / np.linalg.norm(a)


def run_gpu(base, params, nsteps, numelec=2, ms=0):
    import torch
    from sincgpu import SincProject, WalkTables
    sysm, phi, a = base
    n = phi.shape[1]
    with SincProject(11, 0.5, [[0, 0, 0]], [2.0], n, toothnbig=40, toothnsmall=10) as gpu:
        gpu.ci_attach(WalkTables(numelec, n, ms).build_spin())
        gpu.cmf_setup(par_timestep=params.par_timestep, expotol=params.expotol, aerror=params.aerror,
                      aorder=params.aorder, maxaorder=params.maxaorder, expodim=params.expodim,
                      maxexpodim=params.maxexpodim)
        gpu.cmf_pulses(params.pulses)
        e0 = gpu.cmf_init_dev(dev(torch, phi), dev(torch, a))
        steps = [gpu.cmf_step(params.par_timestep * k, params.par_timestep * (k + 1)) for k in range(nsteps)]
        p = torch.empty((n, sysm.G), dtype=torch.complex128, device="cuda")
        av = torch.empty(len(a), dtype=torch.complex128, device="cuda")
        gpu.cmf_state_dev(p, av)
        ez = [gpu.pulse_ez(t) for t in (0.0, 0.013, 0.4, 1.0)]
        steps[-1]["dipole"] = gpu.cmf_dipole_z()
        return e0, steps, host(p), av.cpu().numpy(), ez


def run_oracle(base, params, nsteps):
    sysm, phi, a = base
    o = CmfOracle(sysm, 2, 0, phi, a, params)
    e0 = o.energy
    steps = []
    for k in range(nsteps):
        o.step(params.par_timestep * k, params.par_timestep * (k + 1))
        steps.append({"energy": o.energy, "norm": o.norm, "orb_iters": o.orb_iters, "avec_iters": o.avec_iters})
    steps[-1]["dipole"] = o.dipole()
    return e0, steps, o.s0.spfs, o.s0.avec


@pytest.mark.parametrize("pulsed", [False, True], ids=["field-free", "pulse"])
def test_cmf_steps_match_oracle(base, pulsed):
    pulses = [Pulse(pulsetype=2, omega=2.0, omega2=3.0, strength=0.3)] if pulsed else []
    params = CmfParams(par_timestep=0.01, pulses=pulses)
    e0, steps, phi_g, a_g, ez = run_gpu(base, params, 2)
    e0_r, steps_r, phi_r, a_r = run_oracle(base, params, 2)
    assert e0 == pytest.approx(e0_r, rel=1e-11)
    for s, r in zip(steps, steps_r):
        assert (s["orb_iters"], s["avec_iters"]) == (r["orb_iters"], r["avec_iters"])
        assert s["energy"] == pytest.approx(r["energy"], rel=1e-10)
        assert s["norm"] == pytest.approx(r["norm"], rel=1e-12)
    (d, nn), (d_r, nn_r) = steps[-1]["dipole"], steps_r[-1]["dipole"]
    assert abs(d - d_r) < 1e-9 * max(abs(d_r), 1.0) and nn == pytest.approx(nn_r, rel=1e-12)
    assert np.abs(phi_g - phi_r).max() < 1e-9 * np.abs(phi_r).max()
    assert np.abs(a_g - a_r).max() < 1e-9 * np.abs(a_r).max()
    assert ez == pytest.approx([pulse_ez(pulses, t) for t in (0.0, 0.013, 0.4, 1.0)], abs=1e-15)


def test_cmf_state_stays_normalised_and_orthonormal(base):
    params = CmfParams(par_timestep=0.01)
    _, steps, phi_g, a_g, _ = run_gpu(base, params, 3)
    assert np.abs(np.conj(phi_g).T @ phi_g - np.eye(phi_g.shape[1])).max() < 1e-12
    norms = [s["norm"] for s in steps]
    assert max(norms) - min(norms) < 1e-10          # unitary A-vector propagation


def test_cmf_rejects_misuse(built_lib):
    from sincgpu import SincGpuError, SincProject
    with SincProject(11, 0.5, [[0, 0, 0]], [2.0], 3, toothnbig=40, toothnsmall=10) as gpu:
        with pytest.raises(SincGpuError):
            gpu.cmf_step(0.0, 0.01)                   # no state yet
        with pytest.raises(SincGpuError):
            gpu.cmf_pulses([Pulse(pulsetheta=0.5)])   # transverse polarisation
        with pytest.raises(SincGpuError):
            gpu.cmf_setup(maxaorder=500)
