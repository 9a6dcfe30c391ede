"""Seeded synthetic inputs and the named workloads of the benchmark.

The reference measures on no public dataset; the workloads below are the
synthetic systems of its benchmark configurations, with nuclei snapped to the
grid / half-grid positions the sinc-DVR project requires
(SINCDVR/sincproject.f90:196-204): an odd point count needs even
`centershift` (units of spacing/2).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


@dataclass(frozen=True)
class Workload:
    name: str
    numpoints: int
    spacing: float
    centershift: tuple
    nuccharges: tuple
    nspf: int
    numelec: int
    note: str = ""

    @property
    def G(self):
        return self.numpoints ** 3


WORKLOADS = {
    # He, Z=2 at the origin, 21^3, spacing 0.4, 5 orbitals, 2 electrons (25 configs)
    "A": Workload("A", 21, 0.4, ((0, 0, 0),), (2.0,), 5, 2, "He"),
    # H2-like, Z=1 at z=-+0.75 (centershift +-6 on the 41^3 grid), spacing 0.25, 10 orbitals
    "B": Workload("B", 41, 0.25, ((0, 0, 6), (0, 0, -6)), (1.0, 1.0), 10, 2,
                  "H2-like; nuclei snapped from +-0.7 to +-0.75 bohr (grid parity rule)"),
    # LiH-like, Z=3,1 at z=-+1.5 (centershift +-10), 81^3, spacing 0.3, 16 orbitals, 4 electrons
    "C": Workload("C", 81, 0.3, ((0, 0, 10), (0, 0, -10)), (3.0, 1.0), 16, 4, "LiH-like, 162^3 FFT grid"),
}


def grid_points(numpoints: int, spacing: float) -> np.ndarray:
    p = np.arange(1, numpoints + 1, dtype=np.float64) * spacing
    return p - (p[0] + p[-1]) / 2.0


def seeded_orbitals(numpoints: int, spacing: float, nspf: int, seed: int, width: float = 1.0):
    """phi_k = exp(-|x|^2/(2 w^2)) z_k(x), z ~ CN(0,1) seeded, then modified
    Gram-Schmidt in index order with the hermitian dot.  Shape (G, nspf), Fortran order."""
    rng = np.random.default_rng(seed)
    p = grid_points(numpoints, spacing)
    r2 = p[:, None, None] ** 2 + p[None, :, None] ** 2 + p[None, None, :] ** 2
    G = numpoints ** 3
    env = np.exp(-r2 / (2 * width ** 2)).reshape(G, order="F")
    z = (rng.standard_normal((G, nspf)) + 1j * rng.standard_normal((G, nspf))) / math.sqrt(2)
    out = np.asfortranarray(env[:, None] * z)
    for i in range(nspf):
        for j in range(i):
            out[:, i] -= out[:, j] * np.vdot(out[:, j], out[:, i])
        out[:, i] /= math.sqrt(np.vdot(out[:, i], out[:, i]).real)
    return out


def seeded_avector(numconfig: int, seed: int):
    """A-vector with seeded complex-normal coefficients, normalised."""
    rng = np.random.default_rng(seed)
    a = rng.standard_normal(numconfig) + 1j * rng.standard_normal(numconfig)
    return a / np.linalg.norm(a)


def seeded_hermitian_psd(n: int, seed: int):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    return np.asfortranarray(a @ np.conj(a).T / n + 0.1 * np.eye(n))


def seeded_tally(n: int, seed: int):
    """2-RDM-shaped tally with the symmetries Gamma(a,b,c,d) = conj Gamma(b,a,d,c)
    = Gamma(c,d,a,b)."""
    rng = np.random.default_rng(seed)
    g = rng.standard_normal((n, n, n, n)) + 1j * rng.standard_normal((n, n, n, n))
    g = g + np.conj(g.transpose(1, 0, 3, 2))
    g = g + g.transpose(2, 3, 0, 1)
    return np.asfortranarray(g / 4)


def regularized_inverse(a, tol=1e-10):
    """Host-side helper for synthetic inputs: SVD inverse with the denreg rule."""
    u, s, vt = np.linalg.svd(a)
    inv = np.where(s < tol, 1.0 / tol, 1.0 / np.where(s == 0, 1.0, s))
    inv = np.where(s == 0, 0.0, inv)
    return np.asfortranarray((np.conj(vt).T * inv[None, :]) @ np.conj(u).T)


def snap_shift(z_bohr: float, spacing: float, numpoints: int) -> int:
    """Nuclear coordinate in half-grid units with the project's parity rule:
    an odd point count needs an even shift, an even count an odd one."""
    s = int(round(2.0 * z_bohr / spacing))
    want_odd = numpoints % 2 == 0
    if (s % 2 != 0) != want_odd:
        s += 1 if s >= 0 else -1
    return s


def ci_size(numelec: int, nspf: int) -> int:
    """Determinants of the full CI with the lowest 2Ms."""
    na = (numelec + numelec % 2) // 2
    nb = numelec - na
    return math.comb(nspf, na) * math.comb(nspf, nb)


def _system(rng, nmin, nmax, emin, emax, omin, omax, max_configs):
    N = int(rng.integers(nmin // 2, nmax // 2 + 1)) * 2 + 1          # odd point counts
    spacing = round(float(rng.uniform(0.25, 0.4)), 3)
    ncent = int(rng.integers(1, 3))
    cs, z = [], []
    while len(cs) < ncent:
        pos = rng.uniform(-2.0, 2.0, size=3)
        c = tuple(snap_shift(p, spacing, N) for p in pos)
        if c in cs:          # two nuclei on one point: draw again
            continue
        cs.append(c)
        z.append(float(rng.integers(1, 4)))
    ne = int(rng.integers(emin, emax + 1))
    lo = max(omin, (ne + 1) // 2 + 1)
    n = int(rng.integers(lo, omax + 1))
    while n > lo and max_configs and ci_size(ne, n) > max_configs:
        n -= 1
    return dict(numpoints=N, spacing=spacing, centershift=tuple(cs), nuccharges=tuple(z), nspf=n, numelec=ne,
                restrictms=ne % 2)


def batched_instances(count: int = 64, seed: int = 2024, max_configs: int | None = None):
    """Instances of the batched form: 21^3-61^3 grids (odd point counts),
    spacing 0.25-0.4, 1-2 nuclei of charge 1-3 within +-2 bohr (snapped), 2-6
    electrons, 4-12 orbitals, full CI with the lowest 2Ms (up to C(12,3)^2 =
    48400 determinants); with `max_configs` the orbital count is lowered until
    the full CI has at most that many determinants."""
    rng = np.random.default_rng(seed)
    return [_system(rng, 21, 61, 2, 6, 4, 12, max_configs) for _ in range(count)]


def served_requests(count: int = 24, seed: int = 4048, nmax: int = 41, omax: int = 8, emax: int = 4,
                    max_configs: int = 1000, rate: float = 20.0, nmin: int = 21):
    """Requests of the served form with Poisson arrival offsets (mean `rate`
    per second) and one linearly polarised sin^2 pulse each (peak field
    0.005-0.17 au, carrier 0.05-1.0 au, envelope 400-1600 au; pulse type 2 with
    omega = pi / duration and strength = peak / carrier).  Grids of
    nmin^3-nmax^3 points (odd counts), 2-emax electrons, 4-omax orbitals, the
    orbital count lowered until the full CI has at most `max_configs`
    determinants."""
    rng = np.random.default_rng(seed)
    out, t = [], 0.0
    for _ in range(count):
        t += float(rng.exponential(1.0 / rate))
        s = _system(rng, nmin, nmax, 2, emax, 4, omax, max_configs)
        peak = float(rng.uniform(0.005, 0.17))
        w2 = float(rng.uniform(0.05, 1.0))
        dur = float(rng.uniform(400.0, 1600.0))
        s.update(arrival=t, pulse=dict(pulsetype=2, omega=math.pi / dur, omega2=w2, strength=peak / w2))
        out.append(s)
    return out
