"""The allocation-free Coulomb solve (sincgpu_op_tinv_noalloc_dev).

It exists for callers that cannot call cudaMalloc when they need the solve (a
process whose device memory is partitioned once at start-up, a latency-critical
loop that cannot accept cudaMalloc's synchronisation).  Its scratch is a fixed
device array inside the library; these tests call it through the C ABI and
check it against the regular, allocating op_tinv entry on two calls in a row,
and that a grid too large for the fixed scratch is refused.  This file runs last
(test_zz_*) so that a failure here does not stop the rest of the GPU suite.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-11


def relerr(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("numpoints,spacing,m", [(21, 0.4, 3), (41, 0.25, 12)])
def test_noalloc_matches_regular_entry_twice(built_lib, numpoints, spacing, m):
    import torch
    from sincgpu import SincProject
    from sincgpu.capi import _call, _ptr

    proj = SincProject(numpoints, spacing, [[0, 0, 0]], [1.0], 2)
    try:
        G = numpoints ** 3
        rng = np.random.default_rng(numpoints)
        dens = np.asfortranarray(rng.standard_normal((G, m)) + 1j * rng.standard_normal((G, m)))
        ref = proj.op_tinv(dens)                       # regular entry, allocates its workspace
        d_in = torch.from_numpy(np.ascontiguousarray(dens.T)).cuda()
        d_out = torch.empty_like(d_in)
        for _ in range(2):                             # the scratch keeps the previous call's data
            d_out.fill_(float("nan"))
            torch.cuda.synchronize()
            _call("sincgpu_op_tinv_noalloc_dev", proj._h, _ptr(d_in), _ptr(d_out), m)
            proj.synchronize()
            out = d_out.cpu().numpy().T
            assert np.isfinite(out).all()
            assert relerr(out, ref) < TOL
    finally:
        proj.close()


def test_noalloc_rejects_grid_beyond_fixed_scratch(built_lib):
    import torch
    from sincgpu import SincProject, SincGpuError
    from sincgpu.capi import _call, _ptr

    # 91^3 pads to P=192: one density needs 16*(91*91*192 + 91*192*192) B > 64 MiB
    proj = SincProject(91, 0.3, [[0, 0, 0]], [1.0], 1, toothnsmall=10)
    try:
        assert proj.fft_length == 192
        d = torch.zeros((1, 91 ** 3), dtype=torch.complex128, device="cuda")
        o = torch.empty_like(d)
        with pytest.raises(SincGpuError, match="scratch"):
            _call("sincgpu_op_tinv_noalloc_dev", proj._h, _ptr(d), _ptr(o), 1)
    finally:
        proj.close()


def test_noalloc_fp32_form(built_lib):
    """With coulomb_fp32 (whose FP32 tables are allocated when the option is set,
    not by the call) the entry matches the regular FP32 entry, twice in a row."""
    import torch
    from sincgpu import SincProject
    from sincgpu.capi import _call, _ptr

    N, m = 25, 4
    G = N ** 3
    rng = np.random.default_rng(25)
    dens = np.asfortranarray(rng.standard_normal((G, m)) + 1j * rng.standard_normal((G, m)))
    d_in = torch.from_numpy(np.ascontiguousarray(dens.T)).cuda()
    d_out = torch.empty_like(d_in)
    proj = SincProject(N, 0.4, [[0, 0, 0]], [1.0], 2)
    try:
        proj.set_option("coulomb_fp32", 1)
        for _ in range(2):
            d_out.fill_(float("nan"))
            torch.cuda.synchronize()
            _call("sincgpu_op_tinv_noalloc_dev", proj._h, _ptr(d_in), _ptr(d_out), m)
            proj.synchronize()
            out = d_out.cpu().numpy().T
            assert np.isfinite(out).all()
            ref = proj.op_tinv(dens)                   # regular FP32 entry
            assert relerr(out, ref) < TOL
    finally:
        proj.close()
