"""Generates tests/golden/trajectory_B.npz: 100 field-free constant-mean-field
steps of 0.05 au by the oracle (oracle/cmf_oracle.py: cmf_prop_wfn,
MCTDH.SRC/prop.f90:230-574, with the Expokit A-vector and orbital Krylov
propagators) on the 41^3 workload (two Z=1 nuclei at z=+-0.75 bohr, spacing
0.25, 10 orbitals, 2 electrons, spin-projected singlet), from the seeded
orbitals (sincgpu.inputs.seeded_orbitals seed 1) and A-vector (seeded_avector
seed 2).

The oracle needs about an hour for the 100 steps, so the GPU trajectory test
(tests/test_gpu_trajectory.py) compares against these frozen results.  Stored
per step: energy, norm, the Jacobian and sigma product counts, and the saved
Krylov state of both propagators (orbital Krylov dimension and step size,
A-vector Krylov dimension and step size); at the end: the A-vector, the
orbitals at 512 seeded grid points, their projections onto two seeded weight
vectors over all points, and the z dipole.

    python tests/golden/make_trajectory_b.py [steps]
"""
from __future__ import annotations

import os
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
sys.path.insert(0, str(REPO))
sys.path.insert(0, str(REPO / "v1-1_b200"))

from oracle import sinc_oracle as orc  # noqa: E402
from oracle.cmf_oracle import CmfOracle, CmfParams  # noqa: E402
from oracle.walks_oracle import CIWalks  # noqa: E402
from sincgpu.inputs import WORKLOADS, seeded_avector, seeded_orbitals  # noqa: E402

DT = 0.05


def main(nsteps=100):
    w = WORKLOADS["B"]
    sysm = orc.SincSystem(w.numpoints, w.spacing, w.centershift, w.nuccharges)
    phi = seeded_orbitals(w.numpoints, w.spacing, w.nspf, seed=1)
    a = seeded_avector(CIWalks(w.numelec, w.nspf, 0).numconfig, seed=2)
    o = CmfOracle(sysm, w.numelec, 0, phi, a, CmfParams(par_timestep=DT), workers=os.cpu_count() or 1)
    rec = {k: [] for k in ("energy", "norm", "orb_iters", "avec_iters", "orb_dim", "orb_step", "avec_dim",
                           "avec_step")}
    e0 = o.energy
    t0 = time.time()
    for k in range(nsteps):
        o.step(DT * k, DT * (k + 1))
        for key, v in (("energy", o.energy), ("norm", o.norm), ("orb_iters", o.orb_iters),
                       ("avec_iters", o.avec_iters), ("orb_dim", o.orb.thisexpodim),
                       ("orb_step", o.orb.tempstepsize), ("avec_dim", o.a_dim), ("avec_step", o.a_tempstep)):
            rec[key].append(v)
        print(f"step {k + 1}: E = {o.energy:.15f}, products {o.orb_iters}/{o.avec_iters}, "
              f"{time.time() - t0:.0f} s", flush=True)
    G = w.G
    pts = np.sort(np.random.default_rng(7).choice(G, 512, replace=False))
    rng = np.random.default_rng(8)
    W = rng.standard_normal((G, 2)) + 1j * rng.standard_normal((G, 2))
    d, nn = o.dipole()
    np.savez_compressed(HERE / "trajectory_B.npz", dt=DT, steps=nsteps, energy0=e0,
                        **{k: np.array(v) for k, v in rec.items()}, avector=o.s0.avec, points=pts,
                        phi_pts=o.s0.spfs[pts], phi_proj=W.T @ o.s0.spfs, phi_absmax=np.abs(o.s0.spfs).max(),
                        dipole=d, dipole_norm=nn)
    print(f"written {HERE / 'trajectory_B.npz'}", flush=True)


if __name__ == "__main__":
    main(int(sys.argv[1]) if len(sys.argv) > 1 else 100)
