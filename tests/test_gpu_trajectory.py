"""1000 steps of the 32,768-particle dam break (configs/dam_break_32k.ini:
4 fixed iterations, XSPH, s_corr, the reference's step loop
simulation.c:56-116) on the device, against the FP64 oracle's trajectory
statistics in tests/golden/dam_break_32k_trajectory.json.

The flow is chaotic: single trajectories part after a few hundred steps
whatever the precision, so the device run is held to the spread of the
oracle's own runs with the initial positions moved by uniform +-1e-6
(tests/golden/make_trajectory_envelope.py).  At every checkpoint (every 50
steps) each statistic -- max and mean density error, kinetic energy, centre
of mass -- must lie in the range of the eight oracle runs (unperturbed and
perturbed), widened by that range's own width on each side, plus a floor:
2e-4 of mean density error, 0.5% of kinetic energy, 0.02 length units of
centre of mass, and 10% of the max density error -- the maximum over the
particles is one particle's value, and the oracle's FP32 build already
differs from the FP64 oracle by 7% of it at step 200, before the perturbed
runs have parted.  tests/test_trajectory_band.py checks on the CPU that this
band holds the oracle's FP32 build, an FP32 trajectory of the same
algorithm.
"""
import json
import os

import numpy as np
import pytest

from helpers import parity_record
from sphpc_b200.simulation import Simulation

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                      "dam_break_32k_trajectory.json")

# absolute floors, and relative ones (a fraction of the oracle's value)
FLOOR = {"mean_density_error": 2e-4, "com": 0.02}
REL_FLOOR = {"max_density_error": 0.10, "kinetic_energy": 5e-3}


def band(row, key, axis=None):
    """(low, high) allowed for an FP32 run's value of `key` at one checkpoint."""
    ref = row["oracle"][key]
    lo = row["perturbed_min"][key]
    hi = row["perturbed_max"][key]
    if axis is not None:
        ref, lo, hi = ref[axis], lo[axis], hi[axis]
    lo, hi = min(lo, ref), max(hi, ref)
    width = hi - lo
    floor = FLOOR[key] if key in FLOOR else REL_FLOOR[key] * abs(ref)
    return lo - width - floor, hi + width + floor


def test_dam_break_32k_1000_steps_within_oracle_envelope():
    with open(GOLDEN) as f:
        gold = json.load(f)
    assert gold["config"] == "dam_break_32k" and gold["steps"] == 1000
    every = gold["every"]
    worst = {}
    with Simulation("dam_break_32k") as sim:
        done = 0
        for row in gold["checkpoints"]:
            sim.step(row["step"] - done)
            done = row["step"]
            d = sim.diagnostics()
            for key in ("max_density_error", "mean_density_error", "kinetic_energy"):
                lo, hi = band(row, key)
                assert lo <= d[key] <= hi, (row["step"], key, d[key], lo, hi)
                half = max(hi - lo, 1e-300) / 2
                worst[key] = max(worst.get(key, 0.0), abs(d[key] - (lo + hi) / 2) / half)
            for a in range(3):
                lo, hi = band(row, "com", a)
                assert lo <= d["com"][a] <= hi, (row["step"], "com", a, d["com"][a], lo, hi)
        assert done == gold["steps"]
        assert sim.device_errors() == 0
        final = sim.diagnostics()
    # how far from its band's centre each statistic came, at the worst
    # checkpoint (1 = at the band's edge)
    parity_record("dam_break_32k_1000_steps",
                  {"checkpoints": len(gold["checkpoints"]), "every": every,
                   "worst_fraction_of_band": worst,
                   "final_device": {k: final[k] for k in ("max_density_error",
                                                          "mean_density_error",
                                                          "kinetic_energy")},
                   "final_oracle": {k: gold["checkpoints"][-1]["oracle"][k]
                                    for k in ("max_density_error", "mean_density_error",
                                              "kinetic_energy")}})
    assert np.isfinite(final["kinetic_energy"])
