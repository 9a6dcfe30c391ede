"""Captured-graph and batched forms of the orbital-RHS evaluation.

A captured graph replays exactly the kernels of sincgpu_orbital_rhs_avec_dev,
and a batch launches the graphs of several instances of different sizes at
once; with deterministic reductions every result is bitwise identical to the
direct call, alone or in the batch.  One instance is also checked against the
oracle (1e-11), and the FP32-Coulomb instances of a mixed batch against their
FP64 results (1e-6)."""
import numpy as np
import pytest

from oracle import sinc_oracle as orc
from oracle.walks_oracle import CIWalks

pytestmark = pytest.mark.gpu

INSTANCES = [  # N, spacing, centers, charges, nspf, electrons, 2Ms
    (15, 0.45, [[0, 0, 0]], [2.0], 4, 2, 0),
    (17, 0.4, [[0, 0, 2], [0, 0, -2]], [1.0, 1.0], 5, 2, 0),
    (13, 0.5, [[0, 0, 0]], [3.0], 6, 3, 1),
    (19, 0.35, [[0, 0, 2], [0, 0, -2]], [2.0, 1.0], 5, 4, 0),
]


def make(torch, spec, seed, fp32=False):
    from sincgpu import SincProject, WalkTables
    N, d, cs, z, n, ne, ms = spec
    gpu = SincProject(N, d, cs, z, n)
    wt = WalkTables(ne, n, ms)
    gpu.ci_attach(wt)
    if fp32:
        gpu.set_option("coulomb_fp32", 1)
    G = N ** 3
    sysm = orc.SincSystem(N, d, cs, z)
    phi = orc.seeded_orbitals(sysm, n, seed=seed)
    rng = np.random.default_rng(seed + 1)
    a = rng.standard_normal(wt.numconfig) + 1j * rng.standard_normal(wt.numconfig)
    a /= np.linalg.norm(a)
    cx = dict(dtype=torch.complex128, device="cuda")
    bufs = dict(phi=torch.from_numpy(np.ascontiguousarray(phi.T)).cuda(), a=torch.from_numpy(a).cuda(),
                den=torch.empty((n, n), **cx), inv=torch.empty((n, n), **cx), tally=torch.empty((n,) * 4, **cx),
                mat=torch.empty((n,) * 4, **cx), rp=torch.empty((n, n, G), **cx), out=torch.empty((n, G), **cx))
    return gpu, sysm, phi, a, bufs


def args(b):
    return (b["phi"], b["a"], b["den"], b["inv"], b["tally"], b["mat"], b["rp"], b["out"])


def test_graph_and_batch_are_bitwise_the_direct_call(built_lib):
    import torch
    from sincgpu import Batch
    made = [make(torch, s, 111 + 7 * i) for i, s in enumerate(INSTANCES)]
    direct = []
    for gpu, _, _, _, b in made:
        gpu.orbital_rhs_avec_dev(*args(b))
        torch.cuda.synchronize()
        direct.append(b["out"].clone())
    for (gpu, _, _, _, b), ref in zip(made, direct):
        gpu.rhs_graph_capture(*args(b))
        b["out"].zero_()
        gpu.rhs_graph_launch()
        torch.cuda.synchronize()
        assert torch.equal(b["out"], ref)
    batch = Batch([m[0] for m in made])
    for m in made:
        m[4]["out"].zero_()
    torch.cuda.synchronize()
    batch.launch()
    torch.cuda.synchronize()
    for m, ref in zip(made, direct):
        assert torch.equal(m[4]["out"], ref)
    # one instance against the oracle
    gpu, sysm, phi, a, b = made[0]
    ow = CIWalks(2, 4, 0)
    den = ow.getdenmat00(a)
    inv = orc.invmatsmooth(den)
    _, red = sysm.call_twoe_matel00(phi, phi)
    ref = orc.actreduced00(sysm, phi, phi, den, inv, orc.get_reducedpot(red, ow.get_tworeducedx(a)))
    out = b["out"].cpu().numpy().T
    assert np.abs(out - ref).max() < 1e-11 * np.abs(ref).max()
    batch.close()
    for m in made:
        m[0].close()


def test_mixed_batch_error_and_autotune(built_lib):
    import torch
    from sincgpu import Batch
    plain = [make(torch, s, 211 + 7 * i) for i, s in enumerate(INSTANCES)]
    mixed = [make(torch, s, 211 + 7 * i, fp32=True) for i, s in enumerate(INSTANCES)]
    for (gp, _, _, _, bp), (gm, _, _, _, bm) in zip(plain, mixed):
        gp.orbital_rhs_avec_dev(*args(bp))
        chunk, ms = gm.autotune_rhs(*args(bm))
        assert chunk >= 0 and ms > 0
        # the tuned launch shapes stay in the context
        assert gm.get_option("coul_chunk") == chunk
        assert gm.get_option("twoe_tile") in (0, 4, 5, 6, 7, 8, 9)
        assert gm.get_option("coul_tma") in (-1, 1)
        gm.rhs_graph_capture(*args(bm))
    batch = Batch([m[0] for m in mixed])
    batch.launch()
    torch.cuda.synchronize()
    for (_, _, _, _, bp), (_, _, _, _, bm) in zip(plain, mixed):
        err = float((bm["out"] - bp["out"]).abs().max() / bp["out"].abs().max())
        assert 1e-12 < err < 1e-6
    batch.close()
    for m in plain + mixed:
        m[0].close()
