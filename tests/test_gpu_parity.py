"""Device path (through the C ABI) against the oracle on identical inputs.

Integer work is compared bit for bit: hash keys, the stable sort and its
permutation, cell bounds, neighbour buckets (contents and the reference's
order).  Floating-point stages are compared with the tolerances written in
each test: FP32 device sums against the FP64 oracle.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import assert_close, load_state, oracle_for, oracle_state, rel_err_stats
from sphpc_b200 import _lib
from sphpc_b200.simulation import Simulation

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


def _u32(t):
    return C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_uint))


def _stream():
    return C.c_void_p(_torch().cuda.current_stream().cuda_stream)


# --------------------------------------------------------------------------
# Device-library seam: SortByKey, FindLowerBounds, FindUpperBounds
# --------------------------------------------------------------------------

@pytest.mark.parametrize("n,maxkey,seed", [
    (0, 10, 0), (1, 10, 1), (2, 1, 2), (4095, 1000, 3), (4096, 7, 4), (4097, 100000, 5),
    (100_003, 2 ** 21, 6), (1 << 20, 2 ** 26, 7), (300_000, 2 ** 32 - 1, 8),
    (65_536, 1, 9)])
def test_sort_by_key_stable_bit_exact(n, maxkey, seed):
    torch = _torch()
    rng = np.random.default_rng(seed)
    keys = rng.integers(0, maxkey, size=n, dtype=np.uint64).astype(np.uint32) if maxkey > 1 \
        else np.zeros(n, np.uint32)
    if n >= 2 and maxkey == 2 ** 32 - 1:
        keys[0] = 0xFFFFFFFF
        keys[-1] = 0
    vals = rng.permutation(n).astype(np.uint32)
    dk = torch.from_numpy(keys.view(np.int32)).cuda()
    dv = torch.from_numpy(vals.view(np.int32)).cuda()
    _lib.call("SortByKey", _u32(dk), _u32(dv), n, _stream())
    torch.cuda.synchronize()
    order = np.argsort(keys, kind="stable")
    np.testing.assert_array_equal(dk.cpu().numpy().view(np.uint32), keys[order])
    np.testing.assert_array_equal(dv.cpu().numpy().view(np.uint32), vals[order])


@pytest.mark.parametrize("n,count,seed", [(0, 5, 0), (1, 1, 1), (5000, 1000, 2),
                                           (100_000, 3_000_000, 3), (70_000, 10, 4)])
def test_find_bounds_bit_exact(n, count, seed):
    torch = _torch()
    rng = np.random.default_rng(seed)
    keys = np.sort(rng.integers(0, max(count + 5, 1), size=n).astype(np.uint32))
    dk = torch.from_numpy(keys.view(np.int32)).cuda()
    lo = torch.empty(max(count, 1), dtype=torch.int32, device="cuda")
    hi = torch.empty(max(count, 1), dtype=torch.int32, device="cuda")
    _lib.call("FindLowerBounds", _u32(dk), n, count, _u32(lo), _stream())
    _lib.call("FindUpperBounds", _u32(dk), n, count, _u32(hi), _stream())
    torch.cuda.synchronize()
    c = np.arange(count, dtype=np.uint32)
    np.testing.assert_array_equal(lo.cpu().numpy()[:count].view(np.uint32),
                                  np.searchsorted(keys, c, side="left"))
    np.testing.assert_array_equal(hi.cpu().numpy()[:count].view(np.uint32),
                                  np.searchsorted(keys, c, side="right"))


# --------------------------------------------------------------------------
# Neighbour search: hash, sort, cell ranges, buckets
# --------------------------------------------------------------------------

@pytest.mark.parametrize("config,steps", [("small_dam", 0), ("small_dam", 6),
                                          ("reference_compat", 3)])
def test_find_all_neighbors_bit_exact(config, steps):
    with Simulation(config) as sim:
        sim.step(steps)
        sim.apply_gravity()
        sim.predict_positions()
        sim.find_all_neighbors()
        st = sim.fetch()
        o = oracle_for(sim, st)
        o.call("find_all_neighbors")
        keys, ids, start = sim.cell_data()
        np.testing.assert_array_equal(keys, o.nb_arrays["keys"])
        np.testing.assert_array_equal(ids, o.nb_arrays["ids"])
        Cn = len(o.nb_arrays["start"])
        np.testing.assert_array_equal(start[:Cn], o.nb_arrays["start"])
        np.testing.assert_array_equal(start[1:], np.append(o.nb_arrays["end"], sim.n)[:Cn])
        assert start[Cn] == sim.n
        cnt, nbr = sim.neighbor_buckets()
        ocnt, onbr = o.neighbor_lists()
        np.testing.assert_array_equal(cnt, ocnt)
        for i in range(sim.n):
            np.testing.assert_array_equal(nbr[i, :cnt[i]], onbr[i, :cnt[i]], err_msg=str(i))
        assert sim.device_errors() == 0


def test_find_all_neighbors_bit_exact_with_the_band_open(tmp_path):
    """A box so long (20,000 along x, 10,000 h) that FP32 rounding of its
    largest coordinates could move r^2 across the pre-test band: the host
    then opens the band and every candidate pair is decided by the FP64 test.
    The buckets must still equal the oracle's."""
    from sphpc_b200.scenes import config_path
    text = open(config_path("small_dam")).read().replace("max_x = 48.0", "max_x = 20000.0")
    assert "max_x = 20000.0" in text
    ini = tmp_path / "long_box.ini"
    ini.write_text(text)
    assert not _lib.load().sphpc_neighbor_pretest_fp32_safe(C.c_double(20000.0), C.c_double(2.0))
    with Simulation(str(ini)) as sim:
        sim.step(4)
        sim.apply_gravity()
        sim.predict_positions()
        sim.find_all_neighbors()
        st = sim.fetch()
        o = oracle_for(sim, st)
        o.call("find_all_neighbors")
        cnt, nbr = sim.neighbor_buckets()
        ocnt, onbr = o.neighbor_lists()
        np.testing.assert_array_equal(cnt, ocnt)
        for i in range(sim.n):
            np.testing.assert_array_equal(nbr[i, :cnt[i]], onbr[i, :cnt[i]], err_msg=str(i))
        assert sim.device_errors() == 0


def test_neighbor_cap_60_truncates_in_reference_order():
    """A compressed clump where every particle has more than 60 candidates
    within h: buckets are truncated at 60 in the reference's order."""
    with Simulation("small_dam") as sim:
        st = sim.fetch()
        rng = np.random.default_rng(3)
        n = sim.n
        # squeeze the first 600 particles into a 2.5^3 cube
        for f in ("x", "y", "z"):
            v = st[f].copy()
            v[:600] = 10.0 + 2.5 * rng.random(600)
            st[f] = v
            st[f + "_star"] = v.copy()
        sim.push(st)
        sim.find_all_neighbors()
        st2 = sim.fetch()
        o = oracle_for(sim, st2)
        o.call("find_all_neighbors")
        cnt, nbr = sim.neighbor_buckets()
        ocnt, onbr = o.neighbor_lists()
        assert ocnt.max() == 60
        np.testing.assert_array_equal(cnt, ocnt)
        for i in range(n):
            np.testing.assert_array_equal(nbr[i, :cnt[i]], onbr[i, :cnt[i]])


# --------------------------------------------------------------------------
# Per-stage physics
# --------------------------------------------------------------------------

STAGES = [
    # (device method, oracle function, args, fields, rtol, atol_frac)
    ("compute_densities", "compute_densities", (), ["density"], 1e-5, 0.0),
    ("compute_lambda", "compute_lambda", (), ["lambda"], 1e-4, 1e-5),
    ("update_dps", "update_dps", (0,), ["dp_x", "dp_y", "dp_z"], 1e-4, 1e-5),
    ("update_dps", "update_dps", (2,), ["dp_x", "dp_y", "dp_z"], 1e-4, 1e-5),
    ("update_position_stars", "update_position_stars", (), ["x_star", "y_star", "z_star"],
     1e-6, 0.0),
    ("update_velocities", "update_velocities", (), ["v_x", "v_y", "v_z"], 1e-5, 1e-6),
    ("surface_tension", "surface_tension", (),
     ["color_x", "color_y", "color_z", "v_x", "v_y", "v_z"], 1e-4, 1e-5),
    ("apply_viscosity", "apply_viscosity", (), ["v_x", "v_y", "v_z"], 1e-5, 1e-6),
    ("compute_vorticity", "compute_vorticity", (), ["w_x", "w_y", "w_z"], 1e-4, 1e-4),
    ("vorticity_confinement", "vorticity_confinement", (), ["v_x", "v_y", "v_z"], 1e-5, 1e-6),
    ("update_positions", "update_positions", (), ["x", "y", "z"], 1e-7, 0.0),
]


@pytest.mark.parametrize("config", ["small_dam", "small_obstacle"])
def test_stages_match_oracle(config):
    with Simulation(config) as sim:
        sim.step(8)
        sim.apply_gravity()
        sim.predict_positions()
        sim.find_all_neighbors()
        st = sim.fetch()
        o = oracle_for(sim, st)
        o.call("find_all_neighbors")
        report = {}
        for dev, orc, args, fields, rtol, atol_frac in STAGES:
            st = sim.fetch()
            load_state(o, st)
            o.call(orc, *args)
            getattr(sim, dev)(*args)
            got = sim.fetch()
            want = oracle_state(o)
            for f in fields:
                assert_close(got[f], want[f], rtol, atol_frac, atol=1e-30,
                             what=f"{config}:{dev}{args}:{f}")
                report[f"{dev}{args}:{f}"] = rel_err_stats(got[f], want[f])
        assert sim.device_errors() == 0
        print(report)


# --------------------------------------------------------------------------
# Whole steps
# --------------------------------------------------------------------------

@pytest.mark.parametrize("config", ["small_dam", "small_obstacle", "dam_break_32k"])
def test_one_step_matches_oracle(config):
    """One fused step (sphpc_step) from an evolved state against the FP64
    oracle's step from the same state: positions within 1e-6 relative;
    velocities within 1e-5 relative plus 2e-5 of the velocity scale (the
    FP32 position-correction sums cancel strongly for interior particles)."""
    with Simulation(config) as sim:
        sim.step(5)
        st = sim.fetch()
        o = oracle_for(sim, st)
        sim.step(1)
        o.step(1)
        got = sim.fetch()
        want = oracle_state(o)
        for f in ("x", "y", "z"):
            assert_close(got[f], want[f], 1e-6, 0.0, atol=1e-6, what=f"{config}:{f}")
        for f in ("v_x", "v_y", "v_z"):
            assert_close(got[f], want[f], 1e-5, 2e-5, what=f"{config}:{f}")
        assert_close(got["density"], want["density"], 1e-5, 0.0, what=f"{config}:density")
        assert sim.device_errors() == 0


def test_trajectory_statistics_match_oracle():
    """200 steps of the small dam break: per-step trajectories diverge
    (chaotic flow), the statistics must not: mean density error within 0.05
    percentage points, kinetic energy within 3%, centre of mass within 0.05
    length units at steps 50, 100 and 200; the max density error within 0.5
    percentage points at steps 50 and 100 only.  By step 200 the maximum over
    the particles is itself chaotic: the FP64 oracle alone, with its initial
    positions moved by uniform +-1e-6, ends between 0.75% and 3.6% (mean
    error 5.2e-4 to 6.1e-4, kinetic energy within 1.5%)."""
    with Simulation("small_dam") as sim:
        o = oracle_for(sim)
        done = 0
        for k in (50, 100, 200):
            sim.step(k - done)
            o.step(k - done)
            done = k
            dg = sim.diagnostics()
            do = o.diagnostics()
            if k <= 100:
                assert abs(dg["max_density_error"] - do["max_density_error"]) < 5e-3, (k, dg, do)
            assert abs(dg["mean_density_error"] - do["mean_density_error"]) < 5e-4, (k, dg, do)
            assert abs(dg["kinetic_energy"] / do["kinetic_energy"] - 1) < 0.03, (k, dg, do)
            for a in range(3):
                assert abs(dg["com"][a] - do["com"][a]) < 0.05, (k, dg, do)
        assert sim.device_errors() == 0


# --------------------------------------------------------------------------
# Obstacle
# --------------------------------------------------------------------------

def test_collisions_seam_bit_exact():
    """CalculateParticleCollisions on device double arrays (the reference's
    seam, obstacle_cuda.cu:118-131) against the oracle's restatement."""
    torch = _torch()
    with Simulation("small_obstacle") as sim:
        ob = sim.obstacle
        o = oracle_for(sim)
        rng = np.random.default_rng(11)
        n = 200_000
        pts = [rng.uniform(20.0, 76.0, n), rng.uniform(-1.0, 20.0, n),
               rng.uniform(20.0, 76.0, n)]
        dev = [torch.from_numpy(p.copy()).cuda() for p in pts]
        ptr = [C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_double)) for t in dev]
        _lib.call("CalculateParticleCollisions", ptr[0], ptr[1], ptr[2], n, ob)
        torch.cuda.synchronize()
        want = [p.copy() for p in pts]
        P = C.POINTER(C.c_double)
        o.lib.oracle_particle_collisions(C.byref(o.p), want[0].ctypes.data_as(P),
                                         want[1].ctypes.data_as(P),
                                         want[2].ctypes.data_as(P), n)
        moved = np.sum(want[0] != pts[0])
        assert moved > 1000
        for a in range(3):
            np.testing.assert_array_equal(dev[a].cpu().numpy(), want[a])


def test_obstacle_keeps_particles_out():
    with Simulation("small_obstacle") as sim:
        o = oracle_for(sim)
        sim.step(120)
        st = sim.fetch(["x", "y", "z"])
        import ctypes
        p = o.p
        inside = 0
        for i in range(0, sim.n, 7):
            x, y, z = st["x"][i], st["y"][i], st["z"][i]
            if not (p.ob_min[0] < x < p.ob_max[0] and p.ob_min[1] < y < p.ob_max[1]
                    and p.ob_min[2] < z < p.ob_max[2]):
                continue
            u = np.float32((x - p.ob_min[0]) / np.float32(p.ob_max[0] - p.ob_min[0]))
            v = np.float32((y - p.ob_min[1]) / np.float32(p.ob_max[1] - p.ob_min[1]))
            w = np.float32((z - p.ob_min[2]) / np.float32(p.ob_max[2] - p.ob_min[2]))
            d = o.lib.oracle_sdf_sample(ctypes.byref(p), u, v, w)
            inside += d < -1.0
        assert inside == 0
        assert sim.device_errors() == 0


# --------------------------------------------------------------------------
# Error paths (host-reported, no GPU fault)
# --------------------------------------------------------------------------

def test_stage_before_neighbors_is_an_error():
    with Simulation("small_dam") as sim:
        with pytest.raises(_lib.SphpcError) as e:
            sim.compute_densities()
        assert e.value.code == -5
