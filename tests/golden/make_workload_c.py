"""Generates tests/golden/workload_C.npz: the oracle's results for the 81^3
workload (Z=3 and Z=1 at z=+-1.5 bohr, spacing 0.3, 16 orbitals, 4 electrons,
full M_s=0 CI of 14400 determinants, FFT grid 162^3).

The oracle needs minutes and several GB for this size, so the GPU parity test
(tests/test_gpu_workloads.py) compares against these frozen results instead of
recomputing them.  The inputs are not stored: orbitals and A-vector are seeded
(sincgpu.inputs.seeded_orbitals seed 1, seeded_avector seed 2, the same as
bench.py's rank 0) and regenerated by the test.  What is stored:

* walk tables: per table its length and SHA-256 of the int32 values (the C++
  tables must match bit for bit);
* denmat, invdenmat, the 2-RDM tally, twoematel: complete;
* the orbital RHS at 512 seeded grid points, reducedpot and the reduced
  potentials twoereduced (256 columns each) at every fourth of them, plus
  projections of every grid point onto two seeded complex weight vectors (one
  sum over all 531441 points per column), so that every point enters the
  comparison;
* the one-body matrices (pot, ke, z) and the CI sigma product of the A-vector
  with the matrices assembled from the oracle's twoematel.

    python tests/golden/make_workload_c.py        # about 5 minutes and 10 GB on 8 cores
"""
from __future__ import annotations

import hashlib
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
from oracle.walks_oracle import CIWalks  # noqa: E402
from sincgpu.inputs import WORKLOADS, seeded_avector, seeded_orbitals  # noqa: E402

WALK_TABLES = ["configlist", "numsinglewalks", "numdoublewalks", "singlewalkopspf", "singlewalkdirphase",
               "singlewalk", "doublewalkdirspf", "doublewalkdirphase", "doublewalk", "singlehop_off",
               "singlehop", "singlehopwalkstart", "singlehopwalkend", "doublehop_off", "doublehop",
               "doublehopwalkstart", "doublehopwalkend", "singlediaghop", "doublediaghop"]

NSAMPLE = 512


def table_digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(np.asarray(a), dtype=np.int32).tobytes()).hexdigest()


def sample_points(G: int) -> np.ndarray:
    return np.sort(np.random.default_rng(7).choice(G, NSAMPLE, replace=False))


def weights(G: int) -> np.ndarray:
    rng = np.random.default_rng(8)
    return rng.standard_normal((G, 2)) + 1j * rng.standard_normal((G, 2))


def main():
    w = WORKLOADS["C"]
    workers = os.cpu_count() or 1
    t0 = time.time()
    ow = CIWalks(w.numelec, w.nspf, 0)
    print(f"walks: {ow.numconfig} configs, {time.time() - t0:.0f} s", flush=True)
    digests = {k: table_digest(getattr(ow, k)) for k in WALK_TABLES}
    lengths = {k: int(np.asarray(getattr(ow, k)).size) for k in WALK_TABLES}

    phi = seeded_orbitals(w.numpoints, w.spacing, w.nspf, seed=1)
    a = seeded_avector(ow.numconfig, seed=2)
    den = ow.getdenmat00(a)
    inv = orc.invmatsmooth(den)
    tally = ow.get_tworeducedx(a)
    print(f"rdms: {time.time() - t0:.0f} s", flush=True)

    sysm = orc.SincSystem(w.numpoints, w.spacing, w.centershift, w.nuccharges)
    print(f"tables: {time.time() - t0:.0f} s", flush=True)
    mat, red = sysm.call_twoe_matel00(phi, phi, workers=workers)
    print(f"call_twoe_matel00: {time.time() - t0:.0f} s", flush=True)
    rp = orc.get_reducedpot(red, tally)
    rhs = orc.actreduced00(sysm, phi, phi, den, inv, rp)
    print(f"reducedpot + actreduced00: {time.time() - t0:.0f} s", flush=True)

    G, n = w.G, w.nspf
    pts = sample_points(G)
    W = weights(G)
    red2 = red.reshape(G, n * n, order="F")
    rp2 = rp.reshape(G, n * n, order="F")
    ph = np.conj(phi).T
    pot1 = ph @ sysm.mult_pot(phi)
    ke1 = ph @ sysm.mult_ke(phi)
    z1 = ph @ sysm.mult_zdipole(phi)
    xpot = ow.assemble_doubles(mat)
    xone = ow.assemble_singles(pot1)
    xop = ow.assemble_singles(ke1)
    sigma = ow.sparsesparsemult(a, xpot, xone, xop, constant=sysm.nucrepulsion)
    print(f"sigma: {time.time() - t0:.0f} s", flush=True)

    np.savez_compressed(
        HERE / "workload_C.npz",
        numconfig=ow.numconfig, table_names=np.array(WALK_TABLES),
        table_sha256=np.array([digests[k] for k in WALK_TABLES]),
        table_len=np.array([lengths[k] for k in WALK_TABLES], dtype=np.int64),
        denmat=den, invdenmat=inv, tally=tally, twoematel=mat,
        points=pts, rhs_pts=rhs[pts], points_wide=pts[::4], reducedpot_pts=rp2[pts[::4]],
        twoereduced_pts=red2[pts[::4]],
        rhs_proj=W.T @ rhs, reducedpot_proj=W.T @ rp2, twoereduced_proj=W.T @ red2,
        rhs_absmax=np.abs(rhs).max(), reducedpot_absmax=np.abs(rp).max(), twoereduced_absmax=np.abs(red).max(),
        onebody_pot=pot1, onebody_ke=ke1, onebody_z=z1, nucrepulsion=sysm.nucrepulsion, sigma=sigma)
    print(f"written {HERE / 'workload_C.npz'} after {time.time() - t0:.0f} s", flush=True)


if __name__ == "__main__":
    main()
