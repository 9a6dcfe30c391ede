"""The benchmark's roofline arithmetic (host code, no GPU): the algorithmic bytes
and flops of the Coulomb passes, and the HBM peak's source."""
import json
import math
import sys
from pathlib import Path

REPO = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(REPO))

import bench  # noqa: E402


def test_z_pass_bytes_and_flops_41():
    """41^3 grid, P = 81, 55 pairs: the W2 slab of each pair read and written once
    (2 x 16 N P^2 bytes) plus the real spectrum once per launch (8 P^3)."""
    by, fl = bench.coulomb_pass_work("coul_z", 41, 81, 55)
    assert by == 2 * 16 * 41 * 81 ** 2 * 55 + 8 * 81 ** 3 == 477693288
    assert math.isclose(fl, (2 * 81 ** 2 * 5 * 81 * math.log2(81) + 2 * 81 ** 3) * 55)


def test_pass_bytes_sum_81():
    """81^3 grid, P = 162, 136 pairs: the five passes' floor at 6531 GB/s is 4.79 ms."""
    total = sum(bench.coulomb_pass_work(k, 81, 162, 136)[0]
                for k in ("coul_fwd_x", "coul_fwd_y", "coul_z", "coul_inv_y", "coul_inv_x"))
    assert abs(total / 6531e9 * 1e3 - 4.79) < 0.01


def test_measured_peaks_source(tmp_path, monkeypatch):
    monkeypatch.setattr(bench, "REPO", tmp_path)
    v, src = bench.measured_peaks()
    assert v == 6650.0 and "fallback" in src
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps({"hbm_gbs": 6531.0}))
    v, src = bench.measured_peaks()
    assert v == 6531.0 and "measured" in src


def test_roofline_of_z_pass_81(monkeypatch):
    """The headline workload's z pass (4 launches per evaluation over 136 pairs):
    booked against HBM with the algorithmic bytes of the average launch, and the
    ncu traffic of the 8-pair capture scaled to that launch's 34 pairs."""
    from sincgpu.inputs import WORKLOADS
    monkeypatch.setattr(bench, "_dgemm_tflops", lambda dev: 35.0)
    nprof = 5
    prof = {"coul_z": (4 * 1.2 * nprof, 4 * nprof), "coul_fwd_y": (1.45 * nprof, 4 * nprof)}
    r = bench.make_roofline(WORKLOADS["C"], prof, nprof, None, 162)
    assert r["kernel"] == "coul_z" and r["bound"] == "hbm" and r["launches_per_step"] == 4
    assert r["algorithmic_bytes_per_launch"] == bench.coulomb_pass_work("coul_z", 81, 162, 136)[0] / 4
    assert r["traffic"] == 73350000 * 136 / 4
    assert math.isclose(r["frac"], r["algorithmic_bytes_per_launch"] / 1.2e-3 / 1e9 / r["peak"])
    assert r["fp64"]["bound"] == "fp64"
