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
