"""A 100-step trajectory on the GPU against the oracle's.

100 field-free constant-mean-field steps of 0.05 au (cmf_prop_wfn,
MCTDH.SRC/prop.f90:230-574; Expokit A-vector and orbital Krylov propagators,
MCTDH.SRC/expo_driver.f90:482-1055) on the 41^3 workload (two Z=1 nuclei at
z=+-0.75 bohr, spacing 0.25, 10 orbitals, 2 electrons, spin-projected singlet)
from the seeded orbitals and A-vector that bench.py uses.  The oracle's run
(about an hour on the CPU) is frozen in tests/golden/trajectory_B.npz by
tests/golden/make_trajectory_b.py.

The propagators make discrete decisions (Krylov dimensions, step sizes,
rejected steps: MCTDH.SRC/expo_driver.f90:592-602); every step's Jacobian and
sigma product counts and the orbital propagator's saved Krylov dimension must
equal the oracle's, and its saved step size agree to 1e-9.  Energies and norms
agree to 1e-11 relative at every step; the final A-vector and orbitals to 1e-9
of their largest magnitude (the difference grows slowly along the trajectory
from the 1e-16 rounding differences of each step).
"""
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden" / "trajectory_B.npz"


@pytest.fixture(scope="module")
def traj(built_lib):
    import torch
    from sincgpu import SincProject, WalkTables
    from sincgpu.inputs import WORKLOADS, seeded_avector, seeded_orbitals
    if not GOLDEN.exists():
        pytest.skip("tests/golden/trajectory_B.npz not generated")
    gold = dict(np.load(GOLDEN))
    w = WORKLOADS["B"]
    n, dt, nsteps = w.nspf, float(gold["dt"]), int(gold["steps"])
    phi = seeded_orbitals(w.numpoints, w.spacing, n, seed=1)
    with SincProject(w.numpoints, w.spacing, w.centershift, w.nuccharges, n) as gpu:
        wt = WalkTables(w.numelec, n, 0).build_spin()
        gpu.ci_attach(wt)
        a = seeded_avector(wt.numconfig, seed=2)
        gpu.cmf_setup(par_timestep=dt)
        gpu.cmf_pulses([])
        dphi = torch.from_numpy(np.ascontiguousarray(phi.T)).cuda()
        e0 = gpu.cmf_init_dev(dphi, torch.from_numpy(a).cuda())
        steps = []
        for k in range(nsteps):
            s = gpu.cmf_step(dt * k, dt * (k + 1))
            st = gpu.orbprop_state()
            s["orb_dim"], s["orb_step"] = st["thisexpodim"], st["tempstepsize"]
            steps.append(s)
        p = torch.empty((n, w.G), dtype=torch.complex128, device="cuda")
        av = torch.empty(wt.numconfig, dtype=torch.complex128, device="cuda")
        gpu.cmf_state_dev(p, av)
        d, nn = gpu.cmf_dipole_z()
        out = {"energy0": e0, "steps": steps, "phi": p.cpu().numpy().T, "avector": av.cpu().numpy(),
               "dipole": d, "dipole_norm": nn}
    return gold, out


def test_krylov_decisions_match(traj):
    gold, out = traj
    for k, s in enumerate(out["steps"]):
        assert s["orb_iters"] == gold["orb_iters"][k], f"step {k + 1}"
        assert s["avec_iters"] == gold["avec_iters"][k], f"step {k + 1}"
        assert s["orb_dim"] == gold["orb_dim"][k], f"step {k + 1}"
        assert s["orb_step"] == pytest.approx(gold["orb_step"][k], rel=1e-9), f"step {k + 1}"


def test_energies_and_norms_match(traj):
    gold, out = traj
    assert out["energy0"] == pytest.approx(float(gold["energy0"]), rel=1e-11)
    for k, s in enumerate(out["steps"]):
        assert s["energy"] == pytest.approx(gold["energy"][k], rel=1e-11), f"step {k + 1}"
        assert s["norm"] == pytest.approx(gold["norm"][k], rel=1e-11), f"step {k + 1}"


def test_final_state_matches(traj):
    gold, out = traj
    a_ref = gold["avector"]
    assert np.abs(out["avector"] - a_ref).max() < 1e-9 * np.abs(a_ref).max()
    phi = out["phi"]
    amax = float(gold["phi_absmax"])
    assert np.abs(phi[gold["points"]] - gold["phi_pts"]).max() < 1e-9 * amax
    rng = np.random.default_rng(8)
    W = rng.standard_normal((phi.shape[0], 2)) + 1j * rng.standard_normal((phi.shape[0], 2))
    bound = np.abs(W).sum(axis=0)[:, None] * amax
    assert (np.abs(W.T @ phi - gold["phi_proj"]) / bound).max() < 1e-9
    d_ref = complex(gold["dipole"])
    assert abs(out["dipole"] - d_ref) < 1e-9 * max(abs(d_ref), 1.0)
    # <A|A> = 0.64: the seeded, normalised A-vector loses its non-singlet part in the
    # spin projection at the start and keeps the rest; within the state's 1e-9
    assert out["dipole_norm"] == pytest.approx(float(gold["dipole_norm"]), rel=1e-9)
