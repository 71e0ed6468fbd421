"""Shared test helpers: moving state between the device path (through the C
ABI) and the oracle, and tolerance checks."""
import numpy as np

from oracle.pyoracle import OracleSim, scene_from_ini

# struct Particles field -> oracle state field
FIELD_MAP = {"x_star": "xs", "y_star": "ys", "z_star": "zs", "x": "x", "y": "y", "z": "z",
             "v_x": "vx", "v_y": "vy", "v_z": "vz", "dp_x": "dpx", "dp_y": "dpy",
             "dp_z": "dpz", "w_x": "wx", "w_y": "wy", "w_z": "wz", "color_x": "cx",
             "color_y": "cy", "color_z": "cz", "density": "rho", "lambda": "lam"}


def oracle_for(sim, state=None, fp32=False):
    """An OracleSim with the same scene parameters as `sim` and, when given,
    the device state (a dict from Simulation.fetch())."""
    sc = scene_from_ini(sim.path)
    o = OracleSim(sc, fp32=fp32)
    assert o.n == sim.n, (o.n, sim.n)
    if state is not None:
        load_state(o, state)
    return o


def load_state(o, state):
    for f, of in FIELD_MAP.items():
        if f in state:
            o.a[of][:] = state[f]


def oracle_state(o):
    return {f: o.a[of].copy() for f, of in FIELD_MAP.items()}


def assert_close(got, want, rtol, atol_frac=0.0, atol=0.0, what=""):
    """|got - want| <= rtol*|want| + atol_frac*max|want| + atol, elementwise."""
    got = np.asarray(got, np.float64)
    want = np.asarray(want, np.float64)
    scale = np.max(np.abs(want)) if want.size else 0.0
    tol = rtol * np.abs(want) + atol_frac * scale + atol
    err = np.abs(got - want)
    bad = err > tol
    if np.any(bad):
        i = int(np.argmax(err - tol))
        raise AssertionError(
            f"{what}: {int(bad.sum())}/{bad.size} outside tolerance; worst at {i}: "
            f"got {got[i]!r} want {want[i]!r} (|err| {err[i]:.3e}, tol {tol[i]:.3e}, "
            f"max|want| {scale:.3e})")


def rel_err_stats(got, want):
    got = np.asarray(got, np.float64)
    want = np.asarray(want, np.float64)
    scale = max(np.max(np.abs(want)), 1e-300)
    return float(np.max(np.abs(got - want)) / scale)


def oracle_block(sim, state, lo, hi, idx=None):
    """An OracleSim over the particles of `sim` whose step-start position x
    lies in the box [lo, hi) (three-vectors), or over the given indices, in
    their original order, with the scene's parameters and grid (so hash keys,
    cells and the order within a cell, hence the 60-neighbour cap, are those
    of the whole set).  Returns (oracle, indices of the particles in the
    whole set)."""
    import copy

    x = np.stack([state["x"], state["y"], state["z"]])
    if idx is None:
        inside = np.all((x >= np.asarray(lo)[:, None]) & (x < np.asarray(hi)[:, None]), axis=0)
        idx = np.nonzero(inside)[0]
    sc = copy.copy(scene_from_ini(sim.path))
    sc.x0 = np.ascontiguousarray(x[:, idx])
    o = OracleSim(sc)
    for f, of in FIELD_MAP.items():
        if f in state:
            o.a[of][:] = state[f][idx]
    return o, idx


def interior(state, idx, lo, hi, margin):
    """Mask over idx of the particles at least `margin` inside the box."""
    x = np.stack([state["x"][idx], state["y"][idx], state["z"][idx]])
    lo = np.asarray(lo, np.float64)[:, None] + margin
    hi = np.asarray(hi, np.float64)[:, None] - margin
    return np.all((x >= lo) & (x < hi), axis=0)


def err_stats(got, want, scale=None):
    """Max and median of |got - want| / |want| (relative) and the max of
    |got - want| / max|want| (relative to the field's scale)."""
    got = np.asarray(got, np.float64)
    want = np.asarray(want, np.float64)
    err = np.abs(got - want)
    s = scale if scale is not None else max(float(np.max(np.abs(want))), 1e-300)
    with np.errstate(divide="ignore", invalid="ignore"):
        rel = np.where(want != 0, err / np.abs(want), np.where(err == 0, 0.0, np.inf))
    return {"max_rel": float(np.max(rel)), "median_rel": float(np.median(rel)),
            "max_of_scale": float(np.max(err) / s), "n": int(err.size)}


def parity_record(name, record):
    """Appends one measured-error record to $SPHPC_PARITY_OUT (JSON lines),
    when set, and prints it."""
    import json
    import os

    line = json.dumps({"test": name, **record})
    print("PARITY", line)
    out = os.environ.get("SPHPC_PARITY_OUT")
    if out:
        with open(out, "a") as f:
            f.write(line + "\n")
