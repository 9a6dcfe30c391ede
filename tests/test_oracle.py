"""Pins of the CPU oracle itself (no GPU): committed fixtures, analytic Coulomb
potential, brute-force convolution, dense kinetic operator, symmetries."""
import math
from pathlib import Path

import numpy as np
import pytest

from oracle import sinc_oracle as orc
from oracle.walks_oracle import CIWalks, ci_count

GOLDEN = Path(__file__).resolve().parent / "golden"


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


@pytest.mark.parametrize("name", ["n9", "n7", "n6"])
def test_oracle_matches_committed_fixtures(name):
    g = np.load(GOLDEN / f"sinc_{name}.npz")
    s = orc.SincSystem(int(g["N"]), float(g["spacing"]), g["centershift"], g["charges"],
                       toothnbig=int(g["toothnbig"]), toothnsmall=int(g["toothnsmall"]))
    assert rel(s.tempcoulomb, g["tempcoulomb"]) < 1e-14
    assert rel(s.pot, g["pot"]) < 1e-14
    assert rel(s.op_tinv(g["dens"]), g["optinv"]) < 1e-13
    mat, red = s.call_twoe_matel00(g["phi"], g["phi"])
    assert rel(red, g["twoereduced"]) < 1e-13 and rel(mat, g["twoematel"]) < 1e-13
    rhs = orc.actreduced00(s, g["phi"], g["phi"], g["denmat"], g["invdenmat"], g["reducedpot"], ztdpot=0.02)
    assert rel(rhs, g["rhs"]) < 1e-13


@pytest.mark.parametrize("case", ["2e4o_ms0", "3e4o_ms1", "4e5o_ms0"])
def test_walk_oracle_matches_committed_fixtures(case):
    g = np.load(GOLDEN / f"walks_{case}.npz")
    ne, no, ms = int(case[0]), int(case[2]), int(case.split("ms")[1])
    w = CIWalks(ne, no, ms)
    for k in ("configlist", "singlewalk", "doublewalk", "doublewalkdirspf", "doublewalkdirphase", "doublehop"):
        assert np.array_equal(np.asarray(getattr(w, k)), g[k]), k
    a = g["avector"]
    assert rel(w.getdenmat00(a), g["denmat"]) < 1e-14
    assert rel(w.get_tworeducedx(a), g["tally"]) < 1e-14


def test_gaussian_density_gives_erf_potential():
    """R = T * rho for a normalised Gaussian density approximates erf(r/(sqrt2 s))/r."""
    from scipy.special import erf
    s = orc.SincSystem(21, 0.4, [[0, 0, 0]], [2.0])
    p = s.points
    r = np.sqrt(p[:, None, None] ** 2 + p[None, :, None] ** 2 + p[None, None, :] ** 2)
    sig = 1.0
    rho = (2 * np.pi * sig ** 2) ** -1.5 * np.exp(-r ** 2 / (2 * sig ** 2)) * s.spacing ** 3
    R = s.op_tinv(np.asfortranarray(rho).reshape(-1, 1, order="F"))[:, 0].reshape(21, 21, 21, order="F")
    with np.errstate(divide="ignore", invalid="ignore"):
        V = np.where(r > 0, erf(r / (math.sqrt(2) * sig)) / r, math.sqrt(2 / np.pi) / sig)
    assert np.abs(R.real - V).max() < 5e-5
    assert np.abs(R.imag).max() < 1e-14


def test_doubled_grid_solve_is_the_linear_convolution():
    """op_tinv (2N circular grid, octant embedding/extraction) equals the direct
    sum R(x) = sum_y T(x-y) rho(y): the padded FFT length does not matter."""
    N = 5
    s = orc.SincSystem(N, 0.5, [[0, 0, 0]], [1.0], toothnbig=10, toothnsmall=3)
    rng = np.random.default_rng(0)
    rho = rng.standard_normal((N, N, N)) + 1j * rng.standard_normal((N, N, N))
    T = s.tempcoulomb
    direct = np.zeros((N, N, N), dtype=complex)
    for x in np.ndindex(N, N, N):
        for y in np.ndindex(N, N, N):
            d = tuple(x[k] - y[k] + N - 1 for k in range(3))
            direct[x] += T[d] * rho[y]
    fft = s.op_tinv(np.asfortranarray(rho).reshape(-1, 1, order="F"))[:, 0].reshape(N, N, N, order="F")
    assert rel(fft, direct) < 1e-13


def test_coulomb_kernel_far_field_and_parity():
    s = orc.SincSystem(13, 0.5, [[0, 0, 0]], [1.0], toothnbig=20, toothnsmall=4)
    T = s.tempcoulomb
    assert rel(T, T[::-1, ::-1, ::-1]) < 1e-13            # T(d) = T(-d)
    assert rel(T, np.transpose(T, (1, 0, 2))) < 1e-13     # cubic symmetry
    # beyond toothnsmall the kernel is exactly 1/(spacing |d|) (tooth.f90:141, 83-85)
    d = 12
    assert abs(T[12 + d, 12, 12] * s.spacing * d - 1.0) < 1e-14
    # inside, the near-field correction Q is present
    assert abs(T[12 + 3, 12, 12] * s.spacing * 3 - 1.0) > 1e-6


def test_mult_ke_equals_kronecker_sum():
    N = 4
    s = orc.SincSystem(N, 0.7, [[1, 1, 1]], [1.0], toothnbig=8, toothnsmall=2)
    K = s.ketot
    I = np.eye(N)
    H = np.kron(np.kron(I, I), K.T) + np.kron(np.kron(I, K.T), I) + np.kron(np.kron(K.T, I), I)
    rng = np.random.default_rng(1)
    x = rng.standard_normal((N ** 3, 2)) + 1j * rng.standard_normal((N ** 3, 2))
    assert rel(s.mult_ke(x), H @ x) < 1e-14


def test_twoematel_symmetries():
    s = orc.SincSystem(9, 0.5, [[0, 0, 0]], [1.0], toothnbig=16, toothnsmall=5)
    phi = orc.seeded_orbitals(s, 3, seed=3)
    m, _ = s.call_twoe_matel00(phi, phi)
    assert rel(m, np.conj(m.transpose(1, 0, 3, 2))) < 1e-13   # (a1 b1 a2 b2) -> conj (b1 a1 b2 a2)
    assert rel(m, m.transpose(2, 3, 0, 1)) < 1e-13           # electron exchange (T even)


def test_projected_rhs_is_orthogonal_to_orbitals():
    s = orc.SincSystem(9, 0.5, [[0, 0, 0]], [2.0], toothnbig=16, toothnsmall=5)
    phi = orc.seeded_orbitals(s, 3, seed=4)
    _, red = s.call_twoe_matel00(phi, phi)
    rp = orc.get_reducedpot(red, orc.seeded_tally(3, 5))
    den = orc.seeded_hermitian_psd(3, 6)
    out = orc.actreduced00(s, phi, phi, den, orc.invmatsmooth(den), rp)
    assert np.abs(np.conj(phi).T @ out).max() < 1e-12 * np.abs(out).max()


@pytest.mark.parametrize("ne,n,ms", [(2, 5, 0), (3, 5, 1), (4, 6, 0), (4, 6, 2)])
def test_ci_counts_and_hermitian_sigma(ne, n, ms):
    w = CIWalks(ne, n, ms)
    assert w.numconfig == ci_count(ne, n, ms)
    rng = np.random.default_rng(7)
    tw = rng.standard_normal((n,) * 4) + 1j * rng.standard_normal((n,) * 4)
    tw = tw + np.conj(tw.transpose(1, 0, 3, 2))     # hermitian two-body matrix
    tw = tw + tw.transpose(2, 3, 0, 1)
    h = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    h = h + np.conj(h).T
    xp, xo, xz = w.assemble_doubles(tw), w.assemble_singles(h), w.assemble_singles(0 * h)
    a = rng.standard_normal(w.numconfig) + 1j * rng.standard_normal(w.numconfig)
    b = rng.standard_normal(w.numconfig) + 1j * rng.standard_normal(w.numconfig)
    hab = np.vdot(a, w.sparsesparsemult(b, xp, xo, xz))
    hba = np.vdot(b, w.sparsesparsemult(a, xp, xo, xz))
    assert abs(hab - np.conj(hba)) < 1e-12 * abs(hab)


def test_dgphiv_matches_augmented_exponential():
    """w = exp(tA) v + t phi_1(tA) u equals the top block of
    expm(t [[A, u], [0, 0]]) [v; 1] (Sidje's augmented-matrix identity)."""
    import scipy.linalg as sl
    from oracle.expokit_oracle import dgphiv
    rng = np.random.default_rng(61)
    n = 60
    a = rng.standard_normal((n, n)) / math.sqrt(n)
    a = 0.5 * (a - a.T) + 0.05 * rng.standard_normal((n, n)) / math.sqrt(n)
    u, v = rng.standard_normal(n), rng.standard_normal(n)
    for t, m, guess in ((0.3, 20, 1.0), (2.0, 12, 0.5), (-0.7, 15, 2.0)):
        aug = np.zeros((n + 1, n + 1))
        aug[:n, :n], aug[:n, n] = a, u
        exact = (sl.expm(t * aug) @ np.append(v, 1.0))[:n]
        w, g, info = dgphiv(n, m, t, u, v, 1e-10, 1.0, lambda x: a @ x, lambda x, y: float(x @ y), guess)
        assert np.abs(w - exact).max() < 1e-8 * np.abs(exact).max()
        assert g > 0 and info["nstep"] >= 1


def test_orbital_step_is_orthonormal_and_first_order():
    """expospfprop keeps the orbitals orthonormal and, for a short step, moves
    them by dt * (projected RHS) to first order."""
    from oracle import orbprop_oracle as op
    sysm = orc.SincSystem(9, 0.6, [[0, 0, 0]], [2.0], toothnbig=30, toothnsmall=8)
    n = 3
    phi = orc.seeded_orbitals(sysm, n, seed=62)
    _, red = sysm.call_twoe_matel00(phi, phi)
    tally = orc.seeded_tally(n, seed=63)
    den = orc.seeded_hermitian_psd(n, seed=64)
    slot = (den, orc.invmatsmooth(den), orc.get_reducedpot(red, tally))
    dt = 1e-4
    st = op.OrbPropState(expodim=8, first_stepsize=dt)
    out, info = op.expospfprop(sysm, st, phi, [slot, slot], 0.0, dt, 0.0, dt, True)
    assert np.abs(np.conj(out).T @ out - np.eye(n)).max() < 1e-13
    f = orc.actreduced00(sysm, phi, phi, slot[0], slot[1], slot[2])
    assert np.abs(out - (phi + dt * f)).max() < 50 * dt * dt * np.abs(f).max() ** 2 + 1e-12
    assert info["nstep"] == 1 and info["nmult"] == 1 + 8 + 1
    assert st.icalled == 1 and st.thisexpodim == max(5, math.floor(8 * 0.95))


def test_cmf_step_is_second_order():
    """Field-free energy drift over a fixed time falls like dt^3 per unit time
    (the CMF predictor/corrector scheme is second order)."""
    from oracle.cmf_oracle import CmfOracle, CmfParams
    n = 3
    sysm = orc.SincSystem(9, 0.6, [[0, 0, 0]], [2.0], toothnbig=30, toothnsmall=8)
    phi = orc.seeded_orbitals(sysm, n, seed=93)
    nc = CIWalks(2, n, 0).numconfig
    rng = np.random.default_rng(94)
    a = rng.standard_normal(nc) + 1j * rng.standard_normal(nc)
    drift = []
    for dt in (0.01, 0.005):
        o = CmfOracle(sysm, 2, 0, phi, a / np.linalg.norm(a), CmfParams(par_timestep=dt))
        e0 = o.energy
        for k in range(int(round(0.02 / dt))):
            o.step(dt * k, dt * (k + 1))
        drift.append(abs(o.energy - e0))
    assert drift[1] < drift[0] / 5.0
