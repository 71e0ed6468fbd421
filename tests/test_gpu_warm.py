"""Warm start of the constraint solve on the device: the 16 features and the
training target against the FP64 oracle, and the FP64 residual gate."""
import numpy as np
import pytest

from helpers import assert_close, oracle_for, parity_record
from sphpc_b200 import Simulation
from sphpc_b200 import warm_start as ws

pytestmark = pytest.mark.gpu

# per-feature tolerance: rtol, fraction of the column's max |value|
FEATURE_TOL = {0: (0, 1e-5), 1: (0, 1e-5), 2: (1e-4, 1e-4), 3: (1e-4, 1e-5), 4: (1e-3, 1e-4),
               5: (0, 0), 6: (0, 1e-4), 7: (0, 1e-4), 8: (0, 1e-4), 9: (0, 1e-4),
               10: (0, 1e-4), 11: (0, 1e-4), 12: (1e-5, 1e-5), 13: (1e-5, 1e-6),
               14: (1e-6, 1e-6), 15: (1e-6, 1e-6)}


def _check_features(got, want, what):
    for k, (rtol, frac) in FEATURE_TOL.items():
        assert_close(got[:, k], want[:, k], rtol, frac, atol=1e-7, what=f"{what}: feature {k}")


@pytest.mark.parametrize("config", ["small_dam", "small_obstacle"])
def test_features_match_oracle(config):
    with Simulation(config) as sim:
        sim.step(6)
        st = sim.fetch()
        o = oracle_for(sim, st)
        sim.apply_gravity()
        sim.predict_positions()
        sim.find_all_neighbors()
        got = sim.mlp_features()
        o.call("apply_gravity")
        o.call("predict_positions")
        o.call("find_all_neighbors")
        want = o.features()
        _check_features(got, want, config)
        if config == "small_obstacle":
            assert np.any(want[:, 12] < 4.0)  # some particles inside the obstacle box
        assert sim.device_errors() == 0


@pytest.mark.parametrize("config,iterations", [("small_dam", 4), ("small_obstacle", 6)])
def test_collected_rows_match_oracle(config, iterations):
    """sphpc_mlp_collect: features of the predicted state and the target
    sum_k s_k lambda_k of a plain solve, row for row (rows are in the step's
    cell-sorted order; the step's particle ids map them back)."""
    with Simulation(config) as sim:
        sim.step(4)
        st = sim.fetch()
        o = oracle_for(sim, st)
        ws.dataset_reserve(sim.n)
        ws.dataset_clear()
        rows = ws.collect(sim, iterations)
        assert rows == sim.n and ws.dataset_size() == sim.n
        _, ids, _ = sim.cell_data()
        feat, target = ws.dataset_read(0, sim.n)
        o.call("apply_gravity")
        o.call("predict_positions")
        o.call("find_all_neighbors")
        want_f = o.features()[ids]
        want_t = o.lambda_target(iterations)[ids]
        _check_features(feat, want_f, config)
        assert_close(target, want_t, 1e-3, 1e-3, what=f"{config}: target")
        assert np.all(want_t <= 0.0)
        ws.dataset_free()
        assert sim.device_errors() == 0


def test_gate_discards_a_bad_warm_start():
    """A network whose multipliers are 1000x the first plain ones wrecks the
    warm pass; the FP64 residual gate must discard it and the step must end
    where the plain solver's step ends."""
    solver = {"adaptive": 1, "density_tolerance": 0.002, "max_iterations": 12}
    with Simulation("small_dam", solver) as probe:
        probe.step(5)
        probe.apply_gravity()
        probe.predict_positions()
        probe.find_all_neighbors()
        lam0 = probe.mlp_features()[:, 2]
    params = np.zeros(ws.N_PARAMS, np.float32)
    params[-1] = 1000.0 * float(lam0.min())
    norm = np.concatenate([np.zeros(16), np.ones(16), [1.0]]).astype(np.float32)
    with Simulation("small_dam", solver) as plain, Simulation("small_dam", solver) as warm:
        plain.step(5)
        warm.step(5)
        warm.mlp_load(params, norm)
        warm.set_solver(warm_start=1)
        plain.step(1)
        warm.step(1)
        info = warm.last_step_info()
        assert info["warm_start_used"] == 1 and info["warm_start_rejected"] == 1, info
        p_info = plain.last_step_info()
        assert info["iterations"] == p_info["iterations"] + 1
        got, want = warm.fetch(), plain.fetch()
        for f in ("x", "y", "z"):
            assert_close(got[f], want[f], 1e-6, 0.0, atol=1e-6, what=f"gate:{f}")
        for f in ("v_x", "v_y", "v_z"):
            assert_close(got[f], want[f], 1e-5, 2e-5, what=f"gate:{f}")
        assert warm.device_errors() == 0


def test_trained_network_reduces_iterations():
    """The committed network against the plain solver from the same state:
    early steps of the 4,194,304-particle obstacle scene (seed 0, which the
    training set does not contain), at the scene's tolerance (max density
    error <= 1%), both arms converging every step.  The network in the
    repository takes 2.5 mean iterations here against 2.75 plain."""
    params, norm, meta = ws.load_network()
    solver = {"adaptive": 1, "density_tolerance": 0.01, "max_iterations": 12}
    res = {}
    for arm in ("plain", "warm"):
        with Simulation("obstacle_4m", solver) as sim:
            sim.step(3)
            if arm == "warm":
                sim.mlp_load(params, norm)
                sim.set_solver(warm_start=1, warm_start_scale=meta.get("warm_start_scale", 1.0))
            its, conv = [], 0
            for _ in range(8):
                sim.step(1)
                d = sim.last_step_info()
                its.append(d["iterations"])
                conv += d["converged"]
            assert conv == 8, (arm, its)
            assert sim.device_errors() == 0
            res[arm] = float(np.mean(its))
    print(res)
    assert res["warm"] <= 0.95 * res["plain"], res


def test_network_threshold_skips_mild_steps():
    """warm_start_min_error: a step whose first density pass finds the max
    density error at or below it skips the network, and the next step skips
    the feature pass too (a plain solve); with 0 every step runs the feature
    pass (and the network where the error is above the tolerance)."""
    params, norm, meta = ws.load_network()
    tol = 0.002
    solver = {"adaptive": 1, "density_tolerance": tol, "max_iterations": 12}
    # (plain steps before the network is loaded, threshold)
    for pre, min_error in ((0, 1.0), (5, 1.0), (5, 0.0)):
        with Simulation("small_dam", solver) as sim:
            sim.step(pre)
            sim.mlp_load(params, norm)
            sim.set_solver(warm_start=1, warm_start_min_error=min_error)
            sim.profile(True)
            above, used = 0, 0
            for _ in range(3):
                sim.step(1)
                d = sim.last_step_info()
                above += d["trace"][0] > tol
                used += d["warm_start_used"]
            prof = sim.profile_read()
            features = prof.get("mlp_features", (0, 0.0))[0]
            forward = prof.get("mlp_forward", (0, 0.0))[0]
            if min_error == 0.0:
                assert (features, forward, used) == (3, above, above), (prof, above)
            else:
                # no earlier step: the first step runs the feature pass (and finds
                # a mild step); after that, and after plain steps, none does
                assert (features, forward, used) == (1 if pre == 0 else 0, 0, 0), (pre, prof)
            assert sim.device_errors() == 0


def test_warm_pass_against_plain_iterations_on_config2():
    """The evaluation of the learned warm start on the 1,048,576-particle dam
    break (fixed iteration counts, FP64 residual gate on): from the same state
    60 steps into the collapse, each step's final positions get an extra
    density evaluation, and the mean of the FP64 max density error over 5
    steps is compared between the network's warm pass followed by 2 plain
    iterations and 2, 3 and 4 plain iterations.  The committed network's pass
    is worth one plain iteration here: its arm ends where 3 plain iterations
    end (4.14% and 4.16% over these 5 steps, against 5.07% with 2 and 3.58%
    with 4)."""
    params, norm, meta = ws.load_network()
    err = {}
    for arm, its in (("warm+2", 3), ("plain2", 2), ("plain3", 3), ("plain4", 4)):
        with Simulation("dam_break_1m") as sim:
            sim.step(60)
            if arm == "warm+2":
                sim.mlp_load(params, norm)
                sim.set_solver(warm_start=1, warm_start_min_error=0.0,
                               warm_start_scale=float(meta.get("warm_start_scale", 1.0)))
            # the cap counts every position pass of a step, the warm pass included
            sim.set_solver(solve_iterations=its, adaptive=0)
            e = []
            for _ in range(5):
                sim.step(1)
                if arm == "warm+2":
                    assert sim.last_step_info()["warm_start_used"] == 1
                sim.find_all_neighbors()
                sim.compute_densities()
                e.append(sim.diagnostics()["max_density_error"])
            assert sim.device_errors() == 0
            err[arm] = float(np.mean(e))
    parity_record("warm_pass_vs_plain_iterations_dam_break_1m",
                  {"steps_before": 60, "steps": 5, "mean_max_density_error": err})
    assert err["warm+2"] < 0.9 * err["plain2"], err
    assert err["plain4"] < err["plain3"] < err["plain2"], err
