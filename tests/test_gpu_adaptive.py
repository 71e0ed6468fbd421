"""The adaptive constraint solve: iterate until the FP64 maximum density error
|rho/rho0 - 1| is at most the tolerance, with an iteration cap and the
optional stall stop (solver field min_progress)."""
import numpy as np
import pytest

from helpers import assert_close, oracle_for, oracle_state
from sphpc_b200 import Simulation

pytestmark = pytest.mark.gpu


def test_adaptive_stops_at_the_first_residual_within_tolerance():
    solver = {"adaptive": 1, "density_tolerance": 0.01, "max_iterations": 12}
    with Simulation("small_dam", solver) as sim:
        seen = 0
        for _ in range(12):
            sim.step(1)
            d = sim.last_step_info()
            t = d["trace"]
            if d["converged"]:
                seen += 1
                assert t[-1] <= 0.01 and all(e > 0.01 for e in t[:-1]), d
                assert d["iterations"] == len(t) - 1, d
            else:
                assert d["iterations"] == 12 and all(e > 0.01 for e in t), d
        assert seen > 0
        assert sim.device_errors() == 0


def test_stall_stop_ends_the_solve_without_converging():
    """min_progress p ends the solve at the first density pass k >= 2 whose
    maximum error is not a fraction p below the one two iterations earlier
    (trace[k] > (1 - p) trace[k - 2]); the step is reported as not converged,
    its residual trace is the prefix of the unstopped solve's, and its
    positions are those of the same number of iterations without the stop."""
    cap = 15
    base = {"adaptive": 1, "density_tolerance": 1e-7, "max_iterations": cap}
    with Simulation("small_dam", base) as ref:
        ref.step(8)
        ref.step(1)
        full = ref.last_step_info()["trace"]
    assert len(full) == cap
    ratios = [full[k] / full[k - 2] for k in range(2, cap - 1)]
    p = max(1.0 - max(ratios) + 1e-3, 1e-3)
    stop = next(k for k in range(2, cap - 1) if full[k] > (1.0 - p) * full[k - 2])
    with Simulation("small_dam", base) as sim:
        sim.step(8)
        sim.set_solver(min_progress=p)
        sim.step(1)
        d = sim.last_step_info()
        assert d["converged"] == 0 and d["iterations"] == stop, (d, full, p)
        assert d["trace"] == full[:stop + 1], (d["trace"], full)
        got = sim.fetch()
        assert sim.device_errors() == 0
    with Simulation("small_dam", base) as ref:
        ref.step(8)
        ref.set_solver(max_iterations=stop)
        ref.step(1)
        r = ref.last_step_info()
        assert r["iterations"] == stop and r["converged"] == 0, r
        want = ref.fetch()
    for f in ("x", "y", "z"):
        np.testing.assert_array_equal(got[f], want[f], err_msg=f)


def test_adaptive_step_matches_oracle_at_its_iteration_count():
    """An adaptive step that converges after k position passes ends where the
    FP64 oracle's step of k fixed iterations ends: the same positions, and
    the velocities within a looser bound, since the converged step's post
    passes read the density of its final check (one pass fresher than the
    fixed-iteration step's); with surface tension, whose pair forces scale
    with 2 rho0 / (rho_p + rho_q), that moves a few velocities by up to
    ~1e-4 of the velocity scale."""
    solver = {"adaptive": 1, "density_tolerance": 0.002, "max_iterations": 12}
    for config in ("small_dam", "small_obstacle"):
        with Simulation(config, solver) as sim:
            sim.step(5)
            st = sim.fetch()
            o = oracle_for(sim, st)
            sim.step(1)
            d = sim.last_step_info()
            k = d["iterations"]
            assert d["converged"] == 1 and 1 <= k < 12, d
            o.p.solve_iterations = k
            o.step(1)
            got, want = sim.fetch(), oracle_state(o)
            for f in ("x", "y", "z"):
                assert_close(got[f], want[f], 1e-6, 0.0, atol=1e-6, what=f"{config}:{f}")
            for f in ("v_x", "v_y", "v_z"):
                assert_close(got[f], want[f], 1e-4, 3e-4, what=f"{config}:{f}")
            assert sim.device_errors() == 0
