"""Walk tables: the library's C++ tables must equal the oracle's restatement of
the reference bit for bit (integer indices, phases, order), and match closed-form
counts.  Host code only: runs without a GPU."""
from math import comb

import numpy as np
import pytest

from oracle.walks_oracle import CIWalks, ci_count

TABLES = ["configlist", "numsinglewalks", "numdoublewalks", "singlewalkopspf", "singlewalkdirphase",
          "singlewalk", "doublewalkdirspf", "doublewalkdirphase", "doublewalk", "singlehop_off",
          "singlehop", "singlehopwalkstart", "singlehopwalkend", "doublehop_off", "doublehop",
          "doublehopwalkstart", "doublehopwalkend", "singlediaghop", "doublediaghop"]


@pytest.mark.parametrize("numelec,nspf,ms", [(1, 4, 1), (2, 5, 0), (2, 10, 0), (3, 4, 1), (3, 6, -1),
                                             (4, 5, 0), (4, 6, 2), (4, 7, 0), (5, 5, 1), (6, 6, 0)])
def test_tables_bit_exact(built_lib, numelec, nspf, ms):
    from sincgpu import WalkTables
    o = CIWalks(numelec, nspf, ms)
    w = WalkTables(numelec, nspf, ms, nthreads=3)
    try:
        for name in TABLES:
            a = np.asarray(getattr(o, name))
            b = w.table(name)
            assert a.shape == b.shape, name
            assert np.array_equal(a, b), name
    finally:
        w.close()


def test_thread_count_does_not_change_tables(built_lib):
    from sincgpu import WalkTables
    w1 = WalkTables(4, 8, 0, nthreads=1)
    w2 = WalkTables(4, 8, 0, nthreads=7)
    for name in TABLES:
        assert np.array_equal(w1.table(name), w2.table(name)), name


def test_closed_form_counts_large(built_lib):
    """4 electrons, 16 orbitals, M_s=0: per configuration 60 single walks,
    2*C(16,2)... i.e. 1380 double walks and 1023 double hops."""
    from sincgpu import WalkTables
    w = WalkTables(4, 16, 0)
    assert w.numconfig == ci_count(4, 16, 0) == comb(16, 2) ** 2 == 14400
    assert w.totsinglewalks == 60 * 14400
    assert w.totdoublewalks == 1380 * 14400
    assert w.totdoublehops == 1023 * 14400
    nsw = w.table("numsinglewalks")
    assert np.all(nsw == 60)


def test_walk_invariants(built_lib):
    """Every walk's target exists, phases are +-1, and each config's diagonal hop
    (if any) points back at itself."""
    from sincgpu import WalkTables
    w = WalkTables(4, 7, 0)
    for name in ("singlewalk", "doublewalk"):
        t = w.table(name)
        assert t.min() >= 1 and t.max() <= w.numconfig
    for name in ("singlewalkdirphase", "doublewalkdirphase"):
        assert set(np.unique(w.table(name))) <= {-1, 1}
    off = w.table("doublehop_off")
    hop = w.table("doublehop")
    diag = w.table("doubledaghop") if False else w.table("doublediaghop")
    for c in range(w.numconfig):
        if diag[c] > 0:
            assert hop[off[c] + diag[c] - 1] == c + 1


def test_bad_spin_projection_rejected(built_lib):
    from sincgpu import WalkTables, SincGpuError
    with pytest.raises(SincGpuError):
        WalkTables(4, 6, 1)   # 4 electrons cannot have 2*M_s = 1


def weyl_dim(norb, nelec, two_s):
    """Weyl-Paldus count of spin-adapted configurations (CSFs) with total spin S."""
    s2 = two_s
    return (s2 + 1) * comb(norb + 1, (nelec - s2) // 2) * comb(norb + 1, (nelec + s2) // 2 + 1) // (norb + 1)


@pytest.mark.parametrize("numelec,nspf,ms,two_s", [(2, 4, 0, 0), (2, 4, 0, 2), (3, 4, 1, 1), (3, 4, 1, 3),
                                                   (4, 5, 0, 0), (4, 5, 0, 2), (4, 6, 2, 2), (4, 6, 0, 4),
                                                   (5, 6, -1, 1), (6, 6, 0, 0)])
def test_spin_tables_bit_exact_and_weyl(built_lib, numelec, nspf, ms, two_s):
    """Spin walks, spin sets and eliminated sets match the oracle exactly; the
    projectors agree to rounding; the spin-adapted rank is Weyl's dimension."""
    from oracle.walks_oracle import SpinSets
    from sincgpu import WalkTables
    ow = CIWalks(numelec, nspf, ms)
    sp = SpinSets(ow, two_s)
    wt = WalkTables(numelec, nspf, ms).build_spin(two_s)
    assert wt.numspinconfig == sp.numspinconfig == weyl_dim(nspf, numelec, two_s)
    assert wt.table("numspinwalks").tolist() == [len(x) for x in sp.spinwalk]
    assert wt.table("spinwalk").tolist() == [v for x in sp.spinwalk for v in x]
    assert wt.table("spinwalkdirphase").tolist() == [v for x in sp.spinwalkdirphase for v in x]
    assert wt.table("spinsets").tolist() == [v for st in sp.sets for v in st]
    assert np.diff(wt.table("spinset_off")).tolist() == [len(st) for st in sp.sets]
    assert wt.table("spinsetrank").tolist() == sp.ranks
    assert wt.table("spin_eliminated").tolist() == sp.eliminated
    for p_lib, p_orc in zip(wt.spin_projectors(), sp.projectors):
        assert np.abs(p_lib - p_orc).max() < 1e-13
    wt.close()


def test_spin_projector_is_idempotent_symmetric():
    from oracle.walks_oracle import SpinSets
    sp = SpinSets(CIWalks(4, 6, 0), 2)
    for p in sp.projectors:
        assert np.abs(p @ p - p).max() < 1e-13 and np.abs(p - p.T).max() == 0.0


def test_tables_bit_exact_4e16o_frozen_oracle(built_lib):
    """The 14400-determinant walk tables of the 81^3 / 16-orbital workload
    against the oracle's, frozen as SHA-256 digests of each int32 table in
    tests/golden/workload_C.npz (the pure-Python oracle needs minutes here)."""
    import hashlib
    from pathlib import Path
    from sincgpu import WalkTables
    gold = np.load(Path(__file__).resolve().parent / "golden" / "workload_C.npz")
    w = WalkTables(4, 16, 0)
    try:
        assert w.numconfig == int(gold["numconfig"])
        for name, sha, ln in zip(gold["table_names"], gold["table_sha256"], gold["table_len"]):
            t = np.ascontiguousarray(w.table(str(name)), dtype=np.int32)
            assert t.size == int(ln), name
            assert hashlib.sha256(t.tobytes()).hexdigest() == str(sha), name
    finally:
        w.close()
