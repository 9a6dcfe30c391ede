"""Orbital and A-vector files in the reference's gfortran unformatted layout
(save_vector / write_spf / avector_header_write / write_avector /
easy_load_avectors).  The record reader and writer here are an independent
restatement of the gfortran sequential-record format used to check the
library's bytes."""
import struct

import numpy as np
import pytest

from oracle.walks_oracle import CIWalks, reorder


def records(path):
    out = []
    with open(path, "rb") as f:
        data = f.read()
    i = 0
    while i < len(data):
        (m,) = struct.unpack_from("<i", data, i)
        body = data[i + 4:i + 4 + m]
        (t,) = struct.unpack_from("<i", data, i + 4 + m)
        assert t == m
        out.append(body)
        i += 8 + m
    return out


def write_records(path, bodies):
    with open(path, "wb") as f:
        for b in bodies:
            f.write(struct.pack("<i", len(b)) + b + struct.pack("<i", len(b)))


def test_spf_file_layout_and_round_trip(built_lib, tmp_path):
    from sincgpu.files import load_spfs, save_spfs
    rng = np.random.default_rng(101)
    dims = (5, 4, 3)
    g, n = 60, 3
    phi = np.asfortranarray(rng.standard_normal((g, n)) + 1j * rng.standard_normal((g, n)))
    p = tmp_path / "spfs.bin"
    save_spfs(p, phi, dims)
    rec = records(p)
    assert len(rec) == 2
    assert struct.unpack("<5i", rec[0]) == (5, 4, 3, 3, 1)
    raw = np.frombuffer(rec[1], dtype=np.complex128)
    assert np.array_equal(raw, phi.reshape(-1, order="F"))
    back, d = load_spfs(p)
    assert d == dims and np.array_equal(back, phi)


@pytest.mark.parametrize("numelec,nspf,ms", [(2, 4, 0), (3, 5, 1), (4, 5, 0)])
def test_avector_file_layout_and_round_trip(built_lib, tmp_path, numelec, nspf, ms):
    from sincgpu import WalkTables
    from sincgpu.files import load_avector, save_avector
    wt = WalkTables(numelec, nspf, ms)
    rng = np.random.default_rng(102)
    a = rng.standard_normal((wt.numconfig, 2)) + 1j * rng.standard_normal((wt.numconfig, 2))
    p = tmp_path / "avec.bin"
    save_avector(p, wt, a, allspinproject=1)
    rec = records(p)
    assert struct.unpack("<i", rec[0]) == (2,)
    head = struct.unpack("<100i", rec[1])
    assert head[:7] == (2 * numelec, 1, wt.numconfig, 1, ms, 1, abs(ms)) and not any(head[7:])
    assert struct.unpack("<i", rec[2]) == (1,)
    cl = wt.table("configlist")
    for k in range(wt.numconfig):
        r = rec[3 + k]
        assert list(struct.unpack_from(f"<{2 * numelec}i", r)) == cl[k].tolist()
        assert complex(*struct.unpack_from("<2d", r, 8 * numelec)) == a[k, 0]
    back = load_avector(p, wt, maxvects=2)
    assert np.array_equal(back, a)
    wt.close()


def test_avector_load_reorders_with_phase(built_lib, tmp_path):
    """Determinants stored in another electron order come back with the
    reordering phase (easy_load_avectors)."""
    from sincgpu import WalkTables
    from sincgpu.files import load_avector
    numelec, nspf, ms = 3, 5, 1
    wt = WalkTables(numelec, nspf, ms)
    ow = CIWalks(numelec, nspf, ms)
    rng = np.random.default_rng(103)
    vals = rng.standard_normal(ow.numconfig) + 1j * rng.standard_normal(ow.numconfig)
    bodies = [struct.pack("<i", 1), struct.pack("<100i", 2 * numelec, 1, ow.numconfig, 1, ms, 1, 1, *([0] * 93)),
              struct.pack("<i", 1)]
    expect = np.zeros(ow.numconfig, dtype=np.complex128)
    order = list(range(ow.numconfig))
    rng.shuffle(order)
    for k in order:
        cfg = [int(x) for x in ow.configlist[k]]
        pairs = [cfg[2 * j:2 * j + 2] for j in range(numelec)]
        perm = rng.permutation(numelec)
        shuffled = [v for j in perm for v in pairs[j]]
        phase = reorder(list(shuffled), numelec)
        expect[k] = vals[k] * phase
        bodies.append(struct.pack(f"<{2 * numelec}i", *shuffled) + struct.pack("<2d", vals[k].real, vals[k].imag))
    p = tmp_path / "shuffled.bin"
    write_records(p, bodies)
    got = load_avector(p, wt)[:, 0]
    assert np.array_equal(got, expect)
    wt.close()


def test_avector_load_rejects_foreign_determinant(built_lib, tmp_path):
    from sincgpu import SincGpuError, WalkTables
    from sincgpu.files import load_avector
    wt = WalkTables(2, 3, 0)
    bodies = [struct.pack("<i", 1), struct.pack("<100i", 4, 1, 1, 1, 0, 1, 0, *([0] * 93)), struct.pack("<i", 1),
              struct.pack("<4i", 1, 1, 2, 1) + struct.pack("<2d", 1.0, 0.0)]   # both alpha: Ms = 1
    p = tmp_path / "bad.bin"
    write_records(p, bodies)
    with pytest.raises(SincGpuError):
        load_avector(p, wt)
    wt.close()
