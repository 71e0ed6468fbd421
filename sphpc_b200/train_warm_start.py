"""Generate the warm start's training set with the plain solver and train the
network on the device.

    python -m sphpc_b200.train_warm_start [--out sphpc_b200/weights/warm_start.npz]

Training rows come from the plain PBF solve of two scenes, each with eight
jitter seeds (1-8): the 1,048,576-particle dam break (dam_break_1m) and the
4,194,304-particle obstacle scene with surface tension (obstacle_4m).  Every
scene runs with the adaptive plain solver (max density error <= 1%); the
steps listed in `--collect-at` (early-heavy: the first steps of a dam break
are the most compressed) are taken by sphpc_mlp_collect instead, which solves
with `--iterations` fixed plain substeps and appends one row per particle:
the 16 features of the predicted state and the target
Lambda = sum_k s_k lambda_k.  The network is then trained with AdamW (lr 1e-3
on a half cosine to 1e-5, batch 65,536, ten passes) by the library's
tensor-core kernels, and evaluated on a
collected step of a seed that was not trained on (seed 9); runs of that seed
also choose the multiplier applied to the network's Lambda (0.5, 0.75 or 1:
the fewest mean iterations) and the feature-pass residual below which the
network is skipped (0, 2, 3 or 5 times the tolerance: the shortest run time),
both stored with the network (`--reselect` redoes only these two choices for
an existing network).  The network file
and a JSON log (loss curve, data sizes, held-out fit) are written.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import warm_start as ws
from .simulation import Simulation

SCENES = ("dam_break_1m", "obstacle_4m")


def collect_scene(config, seed, collect_at, iterations, tol, log):
    solver = solver_for(tol, seed)
    rows = 0
    t0 = time.perf_counter()
    with Simulation(config, solver) as sim:
        for k in range(max(collect_at) + 1):
            if k in collect_at:
                rows += ws.collect(sim, iterations)
            else:
                sim.step(1)
        d = sim.diagnostics()
    log(f"  {config} seed {seed}: {rows} rows, {time.perf_counter() - t0:.1f} s, "
        f"final max density error {d['max_density_error']:.4f}")
    return rows


def held_out_fit(params, norm, config, seed, collect_at, iterations, tol):
    """R^2 and relative RMS error of the network on rows of an unseen seed."""
    import ctypes as C
    import torch
    from ._lib import call
    ws.dataset_clear()
    collect_scene(config, seed, collect_at, iterations, tol, lambda *a: None)
    n = ws.dataset_size()
    feat, target = ws.dataset_read(0, n)
    d_feat = torch.from_numpy(feat).cuda()
    d_out = torch.zeros(n, device="cuda")
    F = C.POINTER(C.c_float)
    call("sphpc_mlp_forward", C.c_void_p(d_feat.data_ptr()), n, params.ctypes.data_as(F),
         norm.ctypes.data_as(F), C.c_void_p(d_out.data_ptr()),
         C.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    pred = np.minimum(d_out.cpu().numpy().astype(np.float64), 0.0)
    t = target.astype(np.float64)
    ss_res = np.sum((pred - t) ** 2)
    ss_tot = np.sum((t - t.mean()) ** 2)
    lam0 = feat[:, 2].astype(np.float64)
    # the first plain multiplier, best scaled, as the no-learning baseline
    a = float(lam0 @ t / max(lam0 @ lam0, 1e-300))
    ss_lin = np.sum((a * lam0 - t) ** 2)
    return {"config": config, "seed": seed, "rows": int(n), "r2": float(1 - ss_res / ss_tot),
            "rel_rms": float(np.sqrt(ss_res / max(np.sum(t * t), 1e-300))),
            "baseline_scaled_lambda0_r2": float(1 - ss_lin / ss_tot),
            "baseline_scale": a}


# the solver settings of the comparison the network is chosen for: tolerance
# `tol`, 12 passes at most, the stall stop at 2% over two iterations
def solver_for(tol, seed):
    return {"adaptive": 1, "density_tolerance": tol, "max_iterations": 12, "seed": seed,
            "min_progress": 0.02}


def iterations_with(params, norm, config, seed, scale, pre, steps, tol):
    """Mean constraint iterations per step over `steps` steps after `pre`
    plain steps; scale None = the plain solver."""
    solver = solver_for(tol, seed)
    with Simulation(config, solver) as sim:
        sim.step(pre)
        if scale is not None:
            sim.mlp_load(params, norm)
            sim.set_solver(warm_start=1, warm_start_scale=scale)
        its = []
        for _ in range(steps):
            sim.step(1)
            its.append(sim.last_step_info()["iterations"])
    return float(np.mean(its))


def choose_scale(params, norm, scenes, seed, tol, scales=(0.5, 0.75, 1.0),
                 cases=((3, 8), (150, 8))):
    """The multiplier on the network's Lambda with the fewest iterations on
    held-out runs (seed not trained on), early and later in each scene."""
    table = {}
    for sc in (None,) + tuple(scales):
        tot = 0.0
        for config in scenes:
            for pre, steps in cases:
                it = iterations_with(params, norm, config, seed, sc, pre, steps, tol)
                table[f"{config}@{pre} {'plain' if sc is None else f'x{sc}'}"] = it
                tot += it
        table[f"total {'plain' if sc is None else f'x{sc}'}"] = tot
    best = min(scales, key=lambda s: table[f"total x{s}"])
    return best, table


def seconds_with(params, norm, config, seed, scale, min_error, steps, tol, repeats=2):
    """Device-synchronised seconds of `steps` warm-started steps after 3
    warm-up steps (the fastest of `repeats` runs)."""
    import torch
    best = float("inf")
    for _ in range(repeats):
        with Simulation(config, solver_for(tol, seed)) as sim:
            sim.mlp_load(params, norm)
            sim.set_solver(warm_start=1, warm_start_scale=scale, warm_start_min_error=min_error)
            sim.step(3)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            sim.step(steps)
            torch.cuda.synchronize()
            best = min(best, time.perf_counter() - t0)
    return best


def choose_min_error(params, norm, scenes, seed, tol, scale, factors=(0.0, 2.0, 3.0, 5.0),
                     steps=300):
    """The feature-pass residual below which the network is skipped (a
    multiple of the tolerance), by the run time of held-out runs: a mildly
    compressed step converges in a plain pass or two, which the network's
    cost cannot beat."""
    table = {}
    for f in factors:
        tot = 0.0
        for config in scenes:
            sec = seconds_with(params, norm, config, seed, scale, f * tol, steps, tol)
            table[f"{config} min_error {f:g} tol (s)"] = sec
            tot += sec
        table[f"total min_error {f:g} tol (s)"] = tot
    best = min(factors, key=lambda f: table[f"total min_error {f:g} tol (s)"])
    return best * tol, table


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--out", default=ws.DEFAULT_WEIGHTS)
    ap.add_argument("--log", default=None, help="JSON log (default: next to --out)")
    ap.add_argument("--seeds", type=int, default=8)
    ap.add_argument("--collect-at", default="3,10,40,150,400",
                    help="steps of each scene taken by the collecting solve")
    ap.add_argument("--iterations", type=int, default=2)
    ap.add_argument("--tol", type=float, default=0.01)
    ap.add_argument("--epochs", type=float, default=10.0)
    ap.add_argument("--batch", type=int, default=65536)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--lr-final", type=float, default=1e-5,
                    help="learning rate at the end of the half-cosine schedule")
    ap.add_argument("--weight-decay", type=float, default=1e-4)
    ap.add_argument("--capacity", type=int, default=230_000_000)
    ap.add_argument("--no-held-out", action="store_true")
    ap.add_argument("--scenes", default=",".join(SCENES))
    ap.add_argument("--reselect", action="store_true",
                    help="keep the network in --out and only redo the held-out choices "
                         "(scale, network threshold)")
    args = ap.parse_args(argv)
    logf = args.log or os.path.splitext(args.out)[0] + "_log.json"
    lines = []

    def log(msg):
        print(msg, flush=True)
        lines.append(msg)

    scenes = args.scenes.split(",")
    collect_at = sorted({int(x) for x in args.collect_at.split(",")})
    if args.reselect:
        params, norm, meta = ws.load_network(args.out)
        scale, table = choose_scale(params, norm, scenes, args.seeds + 1, args.tol)
        for k, v in table.items():
            log(f"held-out mean iterations {k}: {v:.2f}")
        min_error, ttable = choose_min_error(params, norm, scenes, args.seeds + 1, args.tol,
                                             scale)
        for k, v in ttable.items():
            log(f"held-out {k}: {v:.3f}")
        log(f"warm-start scale {scale}, network skipped at feature-pass error <= {min_error:g}")
        meta.update({"warm_start_scale": scale, "warm_start_min_error": min_error})
        ws.save_network(args.out, params, norm, meta)
        with open(logf) as fh:
            old = json.load(fh)
        old["meta"] = meta
        old["held_out_iterations"] = table
        old["held_out_seconds"] = ttable
        old["log"] = old.get("log", []) + lines
        with open(logf, "w") as fh:
            json.dump(old, fh, indent=1)
        log(f"rewrote {args.out} and {logf}")
        return
    t0 = time.perf_counter()
    ws.dataset_reserve(args.capacity)
    ws.dataset_clear()
    log(f"collecting: scenes {scenes}, seeds 1-{args.seeds}, collected steps {collect_at}, "
        f"{args.iterations} plain substeps")
    for config in scenes:
        for seed in range(1, args.seeds + 1):
            collect_scene(config, seed, collect_at, args.iterations, args.tol, log)
    n = ws.dataset_size()
    t_collect = time.perf_counter() - t0
    norm = ws.dataset_stats()
    log(f"training set: {n} rows in {t_collect:.1f} s; target std {norm[32]:.4g}")
    steps = int(args.epochs * n / args.batch)
    params = ws.init_params(0)
    t1 = time.perf_counter()
    params, loss = ws.train(params, norm, steps, batch=args.batch, lr=args.lr,
                            weight_decay=args.weight_decay, seed=1, lr_final=args.lr_final)
    t_train = time.perf_counter() - t1
    log(f"trained {steps} AdamW steps of {args.batch} rows in {t_train:.1f} s "
        f"({steps * args.batch / t_train:.3g} rows/s); loss {loss[:10].mean():.4g} -> "
        f"{loss[-100:].mean():.4g}")
    if not np.all(np.isfinite(params)):
        raise SystemExit("training diverged (non-finite parameters)")
    fit = [] if args.no_held_out else [
        held_out_fit(params, norm, c, args.seeds + 1, collect_at, args.iterations, args.tol)
        for c in scenes]
    for f in fit:
        log(f"held-out {f['config']} seed {f['seed']}: R^2 {f['r2']:.4f} (scaled lambda_0: "
            f"{f['baseline_scaled_lambda0_r2']:.4f}), relative RMS {f['rel_rms']:.4f}")
    scale, table = (1.0, {}) if args.no_held_out else choose_scale(
        params, norm, scenes, args.seeds + 1, args.tol)
    for k, v in table.items():
        log(f"held-out mean iterations {k}: {v:.2f}")
    min_error, ttable = (0.0, {}) if args.no_held_out else choose_min_error(
        params, norm, scenes, args.seeds + 1, args.tol, scale)
    for k, v in ttable.items():
        log(f"held-out {k}: {v:.3f}")
    log(f"warm-start scale {scale}, network skipped at feature-pass error <= {min_error:g}")
    meta = {"features": list(ws.FEATURES), "rows": int(n), "steps": steps,
            "warm_start_scale": scale, "warm_start_min_error": min_error,
            "batch": args.batch, "lr": args.lr, "lr_final": args.lr_final,
            "weight_decay": args.weight_decay,
            "scenes": scenes, "seeds": list(range(1, args.seeds + 1)),
            "collected_steps": collect_at,
            "target": f"sum_k s_k lambda_k over {args.iterations} plain substeps"}
    ws.save_network(args.out, params, norm, meta)
    every = max(1, steps // 200)
    with open(logf, "w") as fh:
        json.dump({"meta": meta, "collect_seconds": t_collect, "train_seconds": t_train,
                   "rows_per_second": steps * args.batch / t_train,
                   "loss_every": every, "loss": [float(x) for x in loss[::every]],
                   "held_out": fit, "held_out_iterations": table,
                   "held_out_seconds": ttable, "log": lines}, fh,
                  indent=1)
    ws.dataset_free()
    log(f"wrote {args.out} and {logf}")


if __name__ == "__main__":
    main()
