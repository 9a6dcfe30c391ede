"""Served form: the device-resident request loop.  A request gives bitwise the
same energies and final state alone and in a mix of concurrent requests of
other sizes, the same as the direct CMF entry points, and the loop reports its
step-latency percentiles; admission follows the HBM budget."""
import numpy as np
import pytest

from oracle import sinc_oracle as orc
from oracle.cmf_oracle import Pulse
from oracle.walks_oracle import CIWalks

pytestmark = pytest.mark.gpu

SPECS = [  # N, spacing, centers, charges, nspf, electrons, 2Ms, seed
    (11, 0.5, [[0, 0, 0]], [2.0], 4, 2, 0, 301),
    (13, 0.45, [[0, 0, 2], [0, 0, -2]], [1.0, 1.0], 5, 2, 0, 302),
    (11, 0.5, [[0, 0, 0]], [3.0], 5, 3, 1, 303),
    (15, 0.4, [[0, 0, 0]], [2.0], 4, 2, 0, 304),
    (13, 0.5, [[0, 0, 2], [0, 0, -2]], [2.0, 1.0], 5, 4, 0, 305),
]
PULSE = [Pulse(pulsetype=2, omega=0.5, omega2=1.5, strength=0.05)]


def state(spec):
    N, d, cs, z, n, ne, ms, seed = spec
    sysm = orc.SincSystem(N, d, cs, z)
    phi = orc.seeded_orbitals(sysm, n, seed=seed)
    nc = CIWalks(ne, n, ms).numconfig
    rng = np.random.default_rng(seed + 1)
    a = rng.standard_normal(nc) + 1j * rng.standard_normal(nc)
    return phi, a / np.linalg.norm(a)


_STATES = {}


def submit(srv, spec, nsteps=3, keep=False):
    N, d, cs, z, n, ne, ms, seed = spec
    if seed not in _STATES:
        _STATES[seed] = state(spec)
    phi, a = _STATES[seed]
    return srv.submit(N, d, cs, z, n, ne, ms, phi, a, nsteps, dt=0.01, pulses=PULSE, keep_state=keep)


def prepare(specs):
    """Initial states are built before submitting, so the requests arrive together."""
    for s in specs:
        if s[-1] not in _STATES:
            _STATES[s[-1]] = state(s)


def test_same_alone_and_in_the_mix(built_lib):
    from sincgpu.serve import Server
    prepare(SPECS)
    with Server(max_active=1) as srv:
        alone = srv.wait(submit(srv, SPECS[0], keep=True))
    with Server(max_active=4) as srv:
        ids = [submit(srv, s, keep=(i == 0)) for i, s in enumerate(SPECS)]
        mixed = [srv.wait(i) for i in ids]
        st = srv.stats()
    m = mixed[0]
    assert np.array_equal(m["energies"], alone["energies"])
    assert np.array_equal(m["phi"], alone["phi"]) and np.array_equal(m["avector"], alone["avector"])
    assert st["completed"] == len(SPECS) and st["steps"] == 3 * len(SPECS)
    assert st["peak_active"] >= 2                       # requests overlapped on the device
    assert 0 < st["p50_ms"] <= st["p99_ms"]
    for r in mixed:
        assert abs(r["norm"] - mixed[0]["norm"]) < 1.0 and np.isfinite(r["energy"])


def test_server_equals_direct_cmf(built_lib):
    import torch
    from sincgpu import SincProject, WalkTables
    from sincgpu.serve import Server
    N, d, cs, z, n, ne, ms, _ = SPECS[1]
    phi, a = state(SPECS[1])
    with Server(max_active=2) as srv:
        r = srv.wait(submit(srv, SPECS[1], nsteps=2))
    with SincProject(N, d, cs, z, n) as gpu:
        gpu.ci_attach(WalkTables(ne, n, ms).build_spin())
        gpu.cmf_setup(par_timestep=0.01)
        gpu.cmf_pulses(PULSE)
        e0 = gpu.cmf_init_dev(torch.from_numpy(np.ascontiguousarray(phi.T)).cuda(), torch.from_numpy(a).cuda())
        es = [gpu.cmf_step(0.01 * k, 0.01 * (k + 1))["energy"] for k in range(2)]
    assert r["energy0"] == e0 and list(r["energies"]) == es


def test_admission_by_budget(built_lib):
    from sincgpu.serve import Server
    with Server(max_active=4, hbm_budget=1) as srv:   # nothing fits beside another request
        ids = [submit(srv, s, nsteps=1) for s in SPECS[:3]]
        for i in ids:
            srv.wait(i)
        st = srv.stats()
    assert st["completed"] == 3 and st["peak_active"] == 1
