"""GPU parity at the benchmark's own workloads, through the C ABI.

Workload B (two Z=1 nuclei at z=+-0.75 bohr, 41^3 grid, spacing 0.25, 10
orbitals, 2 electrons, 100 determinants, FFT length 81): the exact call that
bench.py times (sincgpu_orbital_rhs_avec_dev on the same seeded orbitals and
A-vector, the second stream on), so the kernel instances behind its number --
the one-tile symmetric twoematel GEMM (R = 7, 32-point K stages) and the fused
reducedpot + apply kernel (FN = 7) -- are compared with the oracle, computed
once for the module on all host cores.

Workload C (Z=3 and Z=1 at z=+-1.5 bohr, 81^3 grid, spacing 0.3, 16 orbitals,
4 electrons, 14400 determinants, FFT length 162): against the oracle's frozen
results in tests/golden/workload_C.npz (tests/golden/make_workload_c.py; the
oracle takes minutes and GBs at this size).  This runs the multi-tile twoematel
GEMM (2U = 272), the unfused reducedpot GEMM with the separate apply (n > 10),
the 162-point Coulomb passes and the RDM gathers over 14400 determinants.

Tolerance 1e-11 relative to the largest magnitude (the FP64 plain form's bar);
the regularised inverse 1e-10 (it amplifies the denmat's rounding by its
condition number).
"""
import os
from pathlib import Path

import numpy as np
import pytest

from oracle import sinc_oracle as orc
from oracle.walks_oracle import CIWalks

pytestmark = pytest.mark.gpu
TOL = 1e-11
GOLDEN = Path(__file__).resolve().parent / "golden"


def relerr(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


def _run_avec_dev(w, proj, walks, phi_h, a_h):
    """bench.py's timed call on device tensors; returns host copies of every output."""
    import torch
    n, G = w.nspf, w.G
    dev = torch.device("cuda", 0)
    cx = dict(dtype=torch.complex128, device=dev)
    phi = torch.from_numpy(np.ascontiguousarray(phi_h.T)).to(dev)
    avec = torch.from_numpy(np.ascontiguousarray(a_h)).to(dev)
    den, inv = torch.empty((n, n), **cx), torch.empty((n, n), **cx)
    tally, mat = torch.empty((n,) * 4, **cx), torch.empty((n,) * 4, **cx)
    red, out = torch.empty((n, n, G), **cx), torch.empty((n, G), **cx)
    proj.orbital_rhs_avec_dev(phi, avec, den, inv, tally, mat, red, out)
    torch.cuda.synchronize()

    def host(t, shape):
        # torch row-major (.., G) tensors hold the Fortran arrays transposed
        return np.asfortranarray(t.cpu().numpy().T).reshape(shape, order="F")
    return {"denmat": host(den, (n, n)), "invdenmat": host(inv, (n, n)), "tally": host(tally, (n,) * 4),
            "twoematel": host(mat, (n,) * 4), "reducedpot": host(red, (G, n, n)), "rhs": host(out, (G, n))}


# ----------------------------------------------------------------- workload B
@pytest.fixture(scope="module")
def wb(built_lib):
    from sincgpu import SincProject, WalkTables
    from sincgpu.inputs import WORKLOADS, seeded_avector, seeded_orbitals
    w = WORKLOADS["B"]
    phi = seeded_orbitals(w.numpoints, w.spacing, w.nspf, seed=1)
    ow = CIWalks(w.numelec, w.nspf, 0)
    a = seeded_avector(ow.numconfig, seed=2)
    sysm = orc.SincSystem(w.numpoints, w.spacing, w.centershift, w.nuccharges)
    den = ow.getdenmat00(a)
    inv = orc.invmatsmooth(den)
    tally = ow.get_tworeducedx(a)
    mat, red = sysm.call_twoe_matel00(phi, phi, workers=os.cpu_count() or 1)
    rp = orc.get_reducedpot(red, tally)
    ref = {"denmat": den, "invdenmat": inv, "tally": tally, "twoematel": mat, "reducedpot": rp,
           "rhs": orc.actreduced00(sysm, phi, phi, den, inv, rp)}
    proj = SincProject(w.numpoints, w.spacing, w.centershift, w.nuccharges, w.nspf)
    walks = WalkTables(w.numelec, w.nspf, 0)
    proj.ci_attach(walks)
    yield w, proj, walks, phi, a, ref, sysm
    proj.close()


def test_workload_b_benchmarked_call(wb):
    w, proj, walks, phi, a, ref, _ = wb
    assert proj.fft_length == 81
    got = _run_avec_dev(w, proj, walks, phi, a)
    for k in ("denmat", "tally", "twoematel", "reducedpot", "rhs"):
        assert relerr(got[k], ref[k]) < TOL, k
    assert relerr(got["invdenmat"], ref["invdenmat"]) < 1e-10


def test_workload_b_host_entry(wb):
    """The end-to-end call (host orbitals and A-vector in, host RHS out)."""
    w, proj, walks, phi, a, ref, _ = wb
    assert relerr(proj.orbital_rhs_avec(phi, a), ref["rhs"]) < TOL


def test_workload_b_host_entry_upload_groups(wb):
    """The host-array entry copies the orbitals up in groups and starts the
    Coulomb pairs of the first group while the rest is in flight, and copies the
    RHS down while it forms twoematel: the same bits as the device entry for any
    group count (1 = one copy before the evaluation)."""
    w, proj, walks, phi, a, ref, _ = wb
    dev = _run_avec_dev(w, proj, walks, phi, a)["rhs"]
    assert proj.get_option("rhs_upload_groups") == 4
    try:
        for g in (1, 3, 4, 8):
            proj.set_option("rhs_upload_groups", g)
            assert np.array_equal(proj.orbital_rhs_avec(phi, a), dev), g
        proj.set_option("rhs_overlap", 0)
        assert np.array_equal(proj.orbital_rhs_avec(phi, a), dev)
    finally:
        proj.set_option("rhs_overlap", 1)
        proj.set_option("rhs_upload_groups", 4)


def test_workload_b_one_stream_same_bits(wb):
    """rhs_overlap = 0 (the order the per-stage profile uses) gives the same bits."""
    w, proj, walks, phi, a, ref, _ = wb
    o1 = _run_avec_dev(w, proj, walks, phi, a)["rhs"]
    proj.set_option("rhs_overlap", 0)
    try:
        o0 = _run_avec_dev(w, proj, walks, phi, a)["rhs"]
    finally:
        proj.set_option("rhs_overlap", 1)
    assert np.array_equal(o0, o1)


def test_workload_b_reduced_potentials(wb):
    """twoereduced(G, n, n) of all 100 ordered pairs (the 55 hermitian solves mirrored)."""
    w, proj, walks, phi, a, ref, sysm = wb
    mat, red = proj.call_twoe_matel00(phi)
    _, red_ref = sysm.call_twoe_matel00(phi, phi, workers=os.cpu_count() or 1)
    assert relerr(red, red_ref) < TOL
    assert relerr(mat, ref["twoematel"]) < TOL


# ----------------------------------------------------------------- workload C
@pytest.fixture(scope="module")
def wc(built_lib):
    from sincgpu import SincProject, WalkTables
    from sincgpu.inputs import WORKLOADS, seeded_avector, seeded_orbitals
    w = WORKLOADS["C"]
    gold = dict(np.load(GOLDEN / "workload_C.npz"))
    walks = WalkTables(w.numelec, w.nspf, 0)
    assert walks.numconfig == int(gold["numconfig"]) == 14400
    phi = seeded_orbitals(w.numpoints, w.spacing, w.nspf, seed=1)
    a = seeded_avector(walks.numconfig, seed=2)
    proj = SincProject(w.numpoints, w.spacing, w.centershift, w.nuccharges, w.nspf)
    proj.ci_attach(walks)
    got = _run_avec_dev(w, proj, walks, phi, a)
    yield w, proj, walks, phi, a, gold, got
    proj.close()


def _weights(G):
    rng = np.random.default_rng(8)
    return rng.standard_normal((G, 2)) + 1j * rng.standard_normal((G, 2))


def test_workload_c_rdms(wc):
    w, proj, walks, phi, a, gold, got = wc
    assert relerr(got["denmat"], gold["denmat"]) < TOL
    assert relerr(got["tally"], gold["tally"]) < TOL
    assert relerr(got["invdenmat"], gold["invdenmat"]) < 1e-10


def test_workload_c_twoematel(wc):
    w, proj, walks, phi, a, gold, got = wc
    assert proj.fft_length == 162
    assert relerr(got["twoematel"], gold["twoematel"]) < TOL


def test_workload_c_reducedpot_and_rhs(wc):
    """Sampled points (512 for the RHS, 128 for the 256 reducedpot columns) to
    1e-11 of the array's largest magnitude; the weighted sums
    over all 531441 points to 1e-11 of the weights' bound (sum |w| max|x|)."""
    w, proj, walks, phi, a, gold, got = wc
    G, n = w.G, w.nspf
    pts = gold["points"]
    W = _weights(G)
    bound = np.abs(W).sum(axis=0)[:, None]
    rp = got["reducedpot"].reshape(G, n * n, order="F")
    rhs = got["rhs"]
    assert np.abs(rp).max() == pytest.approx(float(gold["reducedpot_absmax"]), rel=1e-11)
    assert np.abs(rhs).max() == pytest.approx(float(gold["rhs_absmax"]), rel=1e-11)
    assert np.abs(rp[gold["points_wide"]] - gold["reducedpot_pts"]).max() < TOL * gold["reducedpot_absmax"]
    assert np.abs(rhs[pts] - gold["rhs_pts"]).max() < TOL * gold["rhs_absmax"]
    assert (np.abs(W.T @ rp - gold["reducedpot_proj"]) / (bound * gold["reducedpot_absmax"])).max() < TOL
    assert (np.abs(W.T @ rhs - gold["rhs_proj"]) / (bound * gold["rhs_absmax"])).max() < TOL


def test_workload_c_host_entry(wc):
    """The end-to-end call at 81^3 (orbitals up in four groups under the Coulomb
    pair loop, the RHS down under twoematel): the device entry's bits."""
    w, proj, walks, phi, a, gold, got = wc
    assert np.array_equal(proj.orbital_rhs_avec(phi, a), got["rhs"])


def test_workload_c_reduced_potentials(wc):
    """twoereduced of all 256 ordered pairs (136 hermitian solves on the 162^3 grid)."""
    import torch
    w, proj, walks, phi, a, gold, got = wc
    G, n = w.G, w.nspf
    cx = dict(dtype=torch.complex128, device="cuda")
    dphi = torch.from_numpy(np.ascontiguousarray(phi.T)).cuda()
    mat = torch.empty((n,) * 4, **cx)
    red = torch.empty((n * n, G), **cx)
    proj.twoe_matel_dev(dphi, dphi, mat, red)
    torch.cuda.synchronize()
    red_h = red.cpu().numpy().T                      # (G, n*n), Fortran pair order
    amax = float(gold["twoereduced_absmax"])
    W = _weights(G)
    bound = np.abs(W).sum(axis=0)[:, None]
    assert np.abs(red_h).max() == pytest.approx(amax, rel=1e-11)
    assert np.abs(red_h[gold["points_wide"]] - gold["twoereduced_pts"]).max() < TOL * amax
    assert (np.abs(W.T @ red_h - gold["twoereduced_proj"]) / (bound * amax)).max() < TOL
    del red
    assert relerr(mat.cpu().numpy().T.reshape((n,) * 4, order="F"), gold["twoematel"]) < TOL


def test_workload_c_sigma(wc):
    """CI sigma over the 14400-determinant walk lists (1023 double hops per
    determinant) with the oracle's matrices assembled on the device."""
    w, proj, walks, phi, a, gold, got = wc
    proj.assemble_sparsemats(gold["twoematel"], gold["onebody_pot"], gold["onebody_ke"], gold["onebody_z"])
    out = proj.sparseconfigmult(a)
    assert relerr(out, gold["sigma"]) < TOL


def test_workload_c_onebody(wc):
    w, proj, walks, phi, a, gold, got = wc
    pot, ke, z = proj.onebody_matel(phi)
    assert relerr(pot, gold["onebody_pot"]) < TOL
    assert relerr(ke, gold["onebody_ke"]) < TOL
    assert relerr(z, gold["onebody_z"]) < TOL
