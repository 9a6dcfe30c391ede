"""GPU (through the C ABI) against the committed golden fixtures: tables, op_tinv,
twoematel/twoereduced, KE, reducedpot, orbital RHS, walk tables, RDMs, sigma."""
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
TOL = 1e-11


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


@pytest.mark.parametrize("name", ["n9", "n7", "n6"])
def test_sinc_fixture(built_lib, name):
    from sincgpu import SincProject
    g = np.load(GOLDEN / f"sinc_{name}.npz")
    n = int(g["nspf"])
    with SincProject(int(g["N"]), float(g["spacing"]), g["centershift"], g["charges"], n,
                     toothnbig=int(g["toothnbig"]), toothnsmall=int(g["toothnsmall"])) as gpu:
        t = gpu.get_tables()
        assert rel(t["tempcoulomb"], g["tempcoulomb"]) < 1e-12
        assert rel(t["pot"], g["pot"]) < 1e-12
        assert rel(gpu.op_tinv(g["dens"]), g["optinv"]) < TOL
        mat, red = gpu.call_twoe_matel00(g["phi"])
        assert rel(red, g["twoereduced"]) < TOL and rel(mat, g["twoematel"]) < TOL
        assert rel(gpu.mult_ke(g["phi"]), g["ke_phi"]) < TOL
        assert rel(gpu.get_reducedpot(g["twoereduced"], g["tally"]), g["reducedpot"]) < TOL
        rhs = gpu.actreduced00(g["phi"], g["phi"], g["denmat"], g["invdenmat"], g["reducedpot"], ztdpot=0.02)
        assert rel(rhs, g["rhs"]) < TOL


@pytest.mark.parametrize("case", ["2e4o_ms0", "3e4o_ms1", "4e5o_ms0"])
def test_walk_fixture(built_lib, case):
    from sincgpu import SincProject, WalkTables
    g = np.load(GOLDEN / f"walks_{case}.npz")
    ne, no, ms = int(case[0]), int(case[2]), int(case.split("ms")[1])
    w = WalkTables(ne, no, ms)
    for k in ("configlist", "singlewalk", "singlewalkopspf", "doublewalk", "doublewalkdirspf",
              "doublewalkdirphase", "doublehop", "doublehopwalkstart", "doublehopwalkend"):
        assert np.array_equal(w.table(k), g[k]), k
    with SincProject(7, 0.6, [[0, 0, 0]], [1.0], no, toothnbig=12, toothnsmall=4) as gpu:
        gpu.ci_attach(w)
        den, _ = gpu.getdenmat(g["avector"])
        assert rel(den, g["denmat"]) < TOL
        assert rel(gpu.get_tworeducedx(g["avector"]), g["tally"]) < TOL
        z = np.zeros((no, no), dtype=np.complex128)
        gpu.assemble_sparsemats(g["twoematel_in"], g["onebody_in"], z, z)
        sig = gpu.sparseconfigmult(g["avector"])
        # the fixture used constant 0.25; this system has one nucleus (no repulsion)
        sig = sig + 0.25 * g["avector"]
        assert rel(sig, g["sigma"]) < TOL
