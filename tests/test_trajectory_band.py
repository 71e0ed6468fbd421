"""The 1000-step trajectory band of tests/test_gpu_trajectory.py, checked on
the CPU against the oracle's FP32 build (tests/golden/
dam_break_32k_trajectory.json, "oracle_fp32"): an FP32 run of the same
algorithm with absolute FP32 coordinates, less precise than the device path,
must stay inside the band the device is held to; and the band must be
narrow enough to mean something (at every checkpoint the kinetic energy
band is within 5% of the oracle's value)."""
import json
import os

from test_gpu_trajectory import GOLDEN, band


def _rows():
    with open(GOLDEN) as f:
        return json.load(f)["checkpoints"]


def test_band_holds_the_fp32_oracle():
    for row in _rows():
        f32 = row["oracle_fp32"]
        for key in ("max_density_error", "mean_density_error", "kinetic_energy"):
            lo, hi = band(row, key)
            assert lo <= f32[key] <= hi, (row["step"], key, f32[key], lo, hi)
        for a in range(3):
            lo, hi = band(row, "com", a)
            assert lo <= f32["com"][a] <= hi, (row["step"], "com", a, f32["com"][a], lo, hi)


def test_band_is_tight():
    for row in _rows():
        ke = row["oracle"]["kinetic_energy"]
        lo, hi = band(row, "kinetic_energy")
        assert hi - lo < 0.10 * ke, (row["step"], lo, hi, ke)
        lo, hi = band(row, "mean_density_error")
        assert hi - lo < 1e-3, (row["step"], lo, hi)


def test_golden_file_is_committed_next_to_its_generator():
    here = os.path.dirname(GOLDEN)
    assert os.path.exists(os.path.join(here, "make_trajectory_envelope.py"))
