"""Checkpoint and resume through the C ABI's host arrays (struct
Particles, the reference's own state): a set saved after k steps and loaded
into a fresh set of the same configuration takes the same next steps as the
run that was not interrupted, bit for bit."""
import numpy as np
import pytest

from sphpc_b200 import Simulation

pytestmark = pytest.mark.gpu

FIELDS = ("x", "y", "z", "v_x", "v_y", "v_z", "density")


@pytest.mark.parametrize("config,solver", [
    ("small_dam", None),                                   # 4 fixed iterations
    ("small_dam", {"adaptive": 1, "density_tolerance": 0.002, "max_iterations": 12}),
])
def test_resume_from_checkpoint_is_bit_exact(tmp_path, config, solver):
    path = str(tmp_path / "state.npz")
    with Simulation(config, solver) as a:
        a.step(10)
        a.save_state(path)
        a.step(10)
        want = a.fetch(FIELDS)
        assert a.device_errors() == 0
    with Simulation(config) as b:
        b.load_state(path)
        b.step(10)
        got = b.fetch(FIELDS)
        assert b.device_errors() == 0
    for f in FIELDS:
        np.testing.assert_array_equal(got[f], want[f], err_msg=f)
