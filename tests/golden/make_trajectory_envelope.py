"""Generates tests/golden/dam_break_32k_trajectory.json: the FP64 oracle's
trajectory statistics of the 32,768-particle dam break (configs/
dam_break_32k.ini, 4 fixed constraint iterations, the reference's step loop
simulation.c:56-116) over 1000 steps, and their spread over runs that
differ by rounding: the initial positions moved by uniform +-1e-6 (seeds
1..7), and runs whose state (x, v) is rounded to FP32 at the end of every
step, as the device stores it (initial perturbation seeds 0..3).  The flow
is chaotic: single trajectories part after a few hundred steps, the
statistics stay within the spread those runs show.  The device run is held to that
spread in tests/test_gpu_trajectory.py.  The same statistics of the
oracle's FP32 build (every `real` a float: what an FP32 trajectory of the
same algorithm does) are stored too; tests/test_trajectory_band.py checks
that the band holds them.

    python tests/golden/make_trajectory_envelope.py     # ~6 min on 8 cores

Test infrastructure: runs only the oracle (oracle/libsphpc_oracle.so).
"""
import json
import multiprocessing as mp
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
CONFIG = "dam_break_32k"
STEPS = 1000
EVERY = 50
SEEDS = [0, 1, 2, 3, 4, 5, 6, 7]   # 0: unperturbed
STORE32 = [100, 101, 102, 103]      # 100 + seed: x, v rounded to FP32 every step
FP32_RUN = -1                       # the FP32 build, unperturbed
PERTURB = 1e-6


def run(seed):
    sys.path.insert(0, ROOT)
    import numpy as np
    from oracle.pyoracle import OracleSim, scene_from_ini
    from sphpc_b200.scenes import config_path
    sc = scene_from_ini(config_path(CONFIG))
    store32 = seed >= 100
    pseed = seed - 100 if store32 else seed
    if pseed > 0:
        rng = np.random.default_rng(pseed)
        sc.x0 = sc.x0 + rng.uniform(-PERTURB, PERTURB, sc.x0.shape)
    o = OracleSim(sc, fp32=(seed == FP32_RUN))
    for f, fs, i in (("x", "xs", 0), ("y", "ys", 1), ("z", "zs", 2)):
        o.a[f][:] = sc.x0[i]
        o.a[fs][:] = sc.x0[i]
    out = []
    for k in range(EVERY, STEPS + 1, EVERY):
        if store32:
            for _ in range(EVERY):
                o.step(1)
                for f in ("x", "y", "z", "vx", "vy", "vz"):
                    o.a[f][:] = o.a[f].astype(np.float32)
                for f, fs in (("x", "xs"), ("y", "ys"), ("z", "zs")):
                    o.a[fs][:] = o.a[f]
        else:
            o.step(EVERY)
        d = o.diagnostics()
        out.append({"step": k, "max_density_error": d["max_density_error"],
                    "mean_density_error": d["mean_density_error"],
                    "kinetic_energy": d["kinetic_energy"], "com": d["com"]})
    return seed, out


def main():
    t0 = time.time()
    ctx = mp.get_context("spawn")
    with ctx.Pool(min(len(SEEDS), os.cpu_count() or 1)) as pool:
        runs = dict(pool.map(run, SEEDS + STORE32 + [FP32_RUN]))
    base = runs[0]
    rows = []
    for i, b in enumerate(base):
        f32 = runs[FP32_RUN][i]
        row = {"step": b["step"], "oracle": {k: b[k] for k in b if k != "step"},
               "oracle_fp32": {k: f32[k] for k in f32 if k != "step"},
               "perturbed_min": {}, "perturbed_max": {}}
        spread = [s for s in SEEDS if s] + STORE32
        for key in ("max_density_error", "mean_density_error", "kinetic_energy"):
            vals = [runs[s][i][key] for s in spread]
            row["perturbed_min"][key] = min(vals)
            row["perturbed_max"][key] = max(vals)
        for a in range(3):
            vals = [runs[s][i]["com"][a] for s in spread]
            row["perturbed_min"].setdefault("com", []).append(min(vals))
            row["perturbed_max"].setdefault("com", []).append(max(vals))
        rows.append(row)
    doc = {"config": CONFIG, "steps": STEPS, "every": EVERY, "perturbation": PERTURB,
           "band": "range of the unperturbed and perturbed runs, widened by its own width "
                   "on each side, plus a floor (tests/test_gpu_trajectory.py)",
           "perturbed_seeds": [s for s in SEEDS if s],
           "fp32_storage_runs": [s - 100 for s in STORE32],
           "generator": "tests/golden/make_trajectory_envelope.py (FP64 oracle)",
           "seconds": round(time.time() - t0, 1), "checkpoints": rows}
    with open(os.path.join(HERE, f"{CONFIG}_trajectory.json"), "w") as f:
        json.dump(doc, f, indent=1)
    print(f"wrote {CONFIG}_trajectory.json in {time.time() - t0:.0f} s")


if __name__ == "__main__":
    main()
