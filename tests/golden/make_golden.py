"""Generates the golden fixtures in this folder from the CPU oracle.

The reference ships no vectors for this path, so these fixtures freeze the
oracle's outputs on small seeded cases; tests compare both the oracle (against
regressions) and the CUDA library (through the C ABI) with them.

    python tests/golden/make_golden.py        # rewrites tests/golden/*.npz
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

from oracle import sinc_oracle as orc  # noqa: E402
from oracle.walks_oracle import CIWalks  # noqa: E402

WALK_TABLES = ["configlist", "numsinglewalks", "numdoublewalks", "singlewalkopspf", "singlewalkdirphase",
               "singlewalk", "doublewalkdirspf", "doublewalkdirphase", "doublewalk", "singlehop_off",
               "singlehop", "singlehopwalkstart", "singlehopwalkend", "doublehop_off", "doublehop",
               "doublehopwalkstart", "doublehopwalkend", "singlediaghop", "doublediaghop"]

# small systems: (name, N, spacing, centershift, charges, toothnbig, toothnsmall, nspf)
SYSTEMS = [
    ("n9", 9, 0.5, [[0, 0, 2]], [1.0], 20, 6, 2),
    ("n7", 7, 0.6, [[0, 0, 0], [2, 0, -2]], [2.0, 1.0], 12, 4, 3),
    ("n6", 6, 0.7, [[1, 1, 1]], [1.0], 10, 3, 2),
]


def sinc_case(name, N, d, cs, z, nbig, nsmall, n):
    s = orc.SincSystem(N, d, cs, z, toothnbig=nbig, toothnsmall=nsmall)
    rng = np.random.default_rng(1000 + N)
    dens = rng.standard_normal((s.G, 2)) + 1j * rng.standard_normal((s.G, 2))
    phi = orc.seeded_orbitals(s, n, seed=2000 + N)
    mat, red = s.call_twoe_matel00(phi, phi)
    tally = orc.seeded_tally(n, seed=3000 + N)
    rp = orc.get_reducedpot(red, tally)
    den = orc.seeded_hermitian_psd(n, seed=4000 + N)
    inv = orc.invmatsmooth(den)
    rhs = orc.actreduced00(s, phi, phi, den, inv, rp, ztdpot=0.02)
    np.savez_compressed(HERE / f"sinc_{name}.npz", N=N, spacing=d, centershift=np.array(cs), charges=np.array(z),
                        toothnbig=nbig, toothnsmall=nsmall, nspf=n, tempcoulomb=s.tempcoulomb, pot=s.pot,
                        kevect=s.kevect, nucrepulsion=s.nucrepulsion, dens=dens, optinv=s.op_tinv(dens),
                        phi=phi, twoematel=mat, twoereduced=red, tally=tally, reducedpot=rp, denmat=den,
                        invdenmat=inv, rhs=rhs, ke_phi=s.mult_ke(phi))


def walk_case(numelec, nspf, ms):
    w = CIWalks(numelec, nspf, ms)
    rng = np.random.default_rng(5000 + 10 * numelec + nspf)
    a = rng.standard_normal(w.numconfig) + 1j * rng.standard_normal(w.numconfig)
    a /= np.linalg.norm(a)
    n = nspf
    tw = rng.standard_normal((n,) * 4) + 1j * rng.standard_normal((n,) * 4)
    h = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    sig = w.sparsesparsemult(a, w.assemble_doubles(tw), w.assemble_singles(h), w.assemble_singles(0 * h),
                             constant=0.25)
    tabs = {k: np.asarray(getattr(w, k)) for k in WALK_TABLES}
    np.savez_compressed(HERE / f"walks_{numelec}e{nspf}o_ms{ms}.npz", avector=a, denmat=w.getdenmat00(a),
                        tally=w.get_tworeducedx(a), twoematel_in=tw, onebody_in=h, sigma=sig, **tabs)


if __name__ == "__main__":
    for case in SYSTEMS:
        sinc_case(*case)
    for case in ((2, 4, 0), (3, 4, 1), (4, 5, 0)):
        walk_case(*case)
    print("written:", sorted(p.name for p in HERE.glob("*.npz")))
