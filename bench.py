#!/usr/bin/env python3
"""Benchmark of the PBF particle pipeline: particle-steps per second on
B200, with the constraint solve iterated until the FP64 max density error is
at most 1% (or the iteration cap).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config NAME]
    python bench.py --impl reference ...   # the reference's own CPU code

One JSON line on stdout (rank 0).  Workload: the 16,777,216-particle full
pipeline scene (configs/full_16m.ini) unless --config says otherwise.  With
N > 1 every rank runs its own replica (the reference path is single rank:
no halo exchange), and `value` is the aggregate over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/sec at max density err <=1%: MLP warm-start vs plain, 1 B200"
UNIT = "particle-steps/s"

# Algorithmic (compulsory) HBM bytes per particle of each stage: every
# particle's own state read and written once in FP32 float4 SoA, neighbour data
# counted once (ideal cache reuse).  The neighbour-list build is not a
# reference-layout stage: x* and cell in, one count byte and ~30 four-byte
# list entries out.
STAGE_BYTES = {
    "hash": 60,                             # r record {x, d} 32, v 16, id 4; w key, slot 4 + 4
    "radix_sort": None,                     # 16 B per digit pass + 4, set below
    "cell_starts": 4,                       # + 8 per cell, added below
    "reorder": 124,                         # r sorted id 4, slot 4, record 32, v 16;
                                            # w record 32, x* 16, neighbour record 16, cell 4
    "build_neighbors": 16 + 4 + 1 + 4 * 30,
    "density_lambda": 24,
    "position": 36,
    "surface_tension": 36 + 68,             # colour + tension
    "xsph": 52,
    "vorticity": 48 + 64,                   # vorticity + confinement
    "velocity": 48,
}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during a region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in (self.out or "").splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": mx or None, "reasons": sorted(reasons), "samples": len(sm)}


def dist_init(args, backend="nccl"):
    """One process per GPU (torchrun's RANK/LOCAL_RANK/WORLD_SIZE); replicas
    only: the process group carries the barriers and the max-over-ranks time,
    no data.  backend "gloo" runs the same host logic on CPU."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        if backend == "nccl":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group(backend, timeout=timedelta(seconds=60))
        pg = dist
    return world, rank, local, pg


def max_over_ranks(value, dist, device):
    """The largest `value` of all ranks (the job's time is its slowest rank's)."""
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world, n, steps, seconds):
    """Whole-job particle-steps/s of `world` replicas of n particles."""
    return world * n * steps / seconds


# --------------------------------------------------------------------------
# CPU reference (the reference's own particles.c / neighbors.c)
# --------------------------------------------------------------------------

class ReferenceSample:
    """The reference's CPU path (oracle/_ref/libsphpc_ref_fast.so: its own
    particles.c and neighbors.c at -O3) on a bounded sample of the workload:
    a 32x32x32 block of the configuration's lattice with its h, dt, box and
    obstacle, stepped with `iterations` constraint iterations."""

    def __init__(self, config_name, iterations, lattice=(32, 32, 32)):
        from oracle.pyoracle import RefSim, scene_from_ini
        from sphpc_b200.scenes import config_path
        sc = scene_from_ini(config_path(config_name))
        nl = sc.meta["lattice"]
        keep = []
        for iz in range(min(lattice[2], nl[2])):
            for iy in range(min(lattice[1], nl[1])):
                base = (iz * nl[1] + iy) * nl[0]
                keep.extend(range(base, base + min(lattice[0], nl[0])))
        sc.x0 = np.ascontiguousarray(sc.x0[:, np.array(keep)])
        self.ref = RefSim(sc, fast=True)
        self.n = sc.n
        self.iterations = iterations
        self.desc = (f"{self.n} particles ({'x'.join(map(str, lattice))} block of "
                     f"{config_name}), {iterations} iterations per step, 1 thread")

    def step_rate(self, steps=1):
        t0 = time.perf_counter()
        self.ref.step(steps, self.iterations)
        return self.n * steps / (time.perf_counter() - t0)


def reference_sample(config_name, iterations, target_s=8.0, max_steps=50):
    rs = ReferenceSample(config_name, iterations)
    rs.step_rate(1)  # warm-up
    steps, t0 = 0, time.perf_counter()
    while steps < max_steps and time.perf_counter() - t0 < target_s:
        rs.ref.step(1, iterations)
        steps += 1
    dt = time.perf_counter() - t0
    return rs.n * steps / dt, {"sample": rs.desc + f", {steps} timed steps", "cores": 1,
                               "kind": "reference"}


def run_reference(args, world, rank):
    if rank != 0:
        return
    rs = ReferenceSample(args.config, args.ref_iterations)
    for _ in range(args.warmup):
        rs.step_rate(1)
    t0 = time.perf_counter()
    rs.ref.step(args.steps, rs.iterations)
    value = rs.n * args.steps / (time.perf_counter() - t0)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "devices": "host CPU, one core (the reference's OpenACC path compiled with gcc has no "
                   "device or multicore target)",
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.config, "sample": rs.desc},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                         "sample": rs.desc},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------
# Our arm
# --------------------------------------------------------------------------

def timed_arm(sim, args, stream, dist, local, dev):
    """W untimed steps, then K steps timed with CUDA events on the launching
    stream between barriers (max over ranks), with the clocks sampled and the
    per-stage CUDA-event profile of the same K steps."""
    import torch
    for _ in range(args.warmup):
        sim.step(1)
    torch.cuda.synchronize()
    sim.profile(True)
    launches0 = sim.launches()
    iters, conv, rejected, used = [], 0, 0, 0
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            sim.step(1)
            if not args.fixed:
                d = sim.last_step_info()
                iters.append(d["iterations"])
                conv += d["converged"]
                used += d["warm_start_used"]
                rejected += d["warm_start_rejected"]
        ev1.record(stream)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
    ms = max_over_ranks(ev0.elapsed_time(ev1), dist, dev)
    prof = sim.profile_read()
    sim.profile(False)
    prof.pop("kernel_launches", None)
    errs = sim.device_errors()
    if errs:
        raise RuntimeError(f"device error bits 0x{errs:x} during the timed region")
    return {"ms": ms, "iters": iters, "converged": conv, "rejected": rejected,
            "warm_used": used, "launches": sim.launches() - launches0,
            "clocks": clk.summary(), "diag": sim.diagnostics(), "prof": prof}


def run_ours(args, world, rank, local, dist):
    import torch
    from sphpc_b200 import Simulation
    from sphpc_b200 import warm_start as ws
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    overrides = {"adaptive": 1, "density_tolerance": args.tol,
                 "max_iterations": args.max_iters, "min_progress": args.min_progress}
    if args.fixed:
        overrides = {"adaptive": 0}
    if args.stiffness_k is not None:
        overrides["stiffness_k"] = args.stiffness_k
    arms = [a.strip() for a in args.arms.split(",") if a.strip()]
    net = None
    warm_settings = None
    if not args.no_warm and os.path.exists(args.weights):
        net = ws.load_network(args.weights)
        # the settings stored with the network unless overridden
        warm_settings = {
            "scale": args.warm_scale if args.warm_scale is not None
            else float(net[2].get("warm_start_scale", 1.0)),
            "min_error": args.warm_min_error if args.warm_min_error is not None
            else float(net[2].get("warm_start_min_error", 0.0)),
            "gate": int(args.warm_gate)}
    stream = torch.cuda.current_stream(dev)

    def make_sim(kind):
        """kind: "plain", "warm" (the network's multipliers) or "carry" (the
        previous step's applied multipliers, no network: the control arm)."""
        t_init = time.perf_counter()
        sim = Simulation(args.config, solver_overrides=overrides)
        sim.set_stream(stream.cuda_stream)
        if kind == "warm":
            sim.mlp_load(net[0], net[1])
            sim.set_solver(warm_start=1, warm_start_source=0,
                           warm_start_scale=warm_settings["scale"],
                           warm_start_min_error=warm_settings["min_error"],
                           warm_start_gate=warm_settings["gate"])
        elif kind == "carry":
            sim.set_solver(warm_start=1, warm_start_source=1, warm_start_min_error=0.0)
        elif kind == "fixed":
            # the reference arm's own iteration count, fixed: the like-for-like
            # comparison with its CPU path
            sim.set_solver(adaptive=0, solve_iterations=args.ref_iterations)
        log(f"[rank {rank}] {args.config}: {sim.n} particles, arm {kind}, "
            f"init {time.perf_counter()-t_init:.1f}s")
        return sim

    # plain solver first, then the network-started one (with a trained
    # network) and the carried-multiplier control, each from the same state
    results = {}
    sim = None
    n = None
    for kind in ["plain"] + [k for k in arms if k != "plain"]:
        if kind == "warm" and net is None:
            continue
        if sim is not None:
            sim.close()
        sim = make_sim(kind)
        n = sim.n
        results[kind] = timed_arm(sim, args, stream, dist, local, dev)
    plain = results["plain"]
    warm = results.get("warm")
    carry = results.get("carry")
    fixed = results.get("fixed")
    head = warm if warm is not None else plain
    ms_max = head["ms"]
    value = job_rate(world, n, args.steps, ms_max / 1e3)
    iters = head["iters"]
    conv = head["converged"]
    launches = head["launches"]
    diag = head["diag"]

    # per-stage CUDA-event profile of the headline arm's timed steps
    prof = head["prof"]

    roof = None
    if prof:
        name, (cnt, tot) = max(prof.items(), key=lambda kv: kv[1][1])
        per = STAGE_BYTES.get(name)
        if name == "radix_sort":
            per = 16 * sim_passes(sim) + 4
        if name == "cell_starts":
            per = 4 + 8 * sim_cells(sim) / n
        if per is not None and cnt:
            avg_s = tot / cnt / 1e3
            bytes_launch = per * n
            peak, kind = peaks()
            achieved = bytes_launch / avg_s / 1e9
            roof = {"kernel": name, "bound": "hbm", "achieved": achieved, "peak": peak,
                    "peak_kind": kind, "unit": "GB/s", "frac": achieved / peak,
                    "traffic": ncu_traffic(name, n), "bytes_per_particle": per,
                    # the neighbour passes are bound by instruction issue, not
                    # by HBM: the share of cycles their schedulers issued
                    "issue_active_ncu": ncu_stage(name).get("issue_active_pct"),
                    "avg_launch_ms": tot / cnt}

    # the HBM-bound stages (hash, sort, cell starts, reorder), each against
    # the measured copy bandwidth on its algorithmic bytes
    hbm_class = {}
    if prof:
        peak, kind = peaks()
        for name in ("hash", "radix_sort", "cell_starts", "reorder"):
            if name not in prof or not prof[name][0]:
                continue
            cnt, tot = prof[name]
            per = STAGE_BYTES[name]
            if name == "radix_sort":
                per = 16 * sim_passes(sim) + 4
            if name == "cell_starts":
                per = 4 + 8 * sim_cells(sim) / n
            gbs = per * n / (tot / cnt / 1e3) / 1e9
            hbm_class[name] = {"bytes_per_particle": per, "avg_launch_ms": tot / cnt,
                               "achieved_gbs": gbs, "frac": gbs / peak}

    # every neighbour stage against the same HBM peak on its algorithmic
    # bytes, beside its committed ncu DRAM bytes and issue activity (these
    # stages are bound by instruction issue and the L1 gathers, not by HBM)
    nbr_stages = {}
    if prof:
        peak, kind = peaks()
        for name in ("build_neighbors", "density_lambda", "position", "surface_tension", "xsph",
                     "vorticity"):
            if name not in prof or not prof[name][0]:
                continue
            cnt, tot = prof[name]
            per = STAGE_BYTES[name]
            gbs = per * n / (tot / cnt / 1e3) / 1e9
            e = ncu_stage(name)
            nbr_stages[name] = {"bytes_per_particle": per, "avg_launch_ms": tot / cnt,
                                "launches_per_step": cnt / args.steps, "achieved_gbs": gbs,
                                "frac": gbs / peak,
                                "dram_bytes_per_particle_ncu": e.get("bytes_per_particle"),
                                "issue_active_ncu": e.get("issue_active_pct")}

    # end to end through the C ABI with host buffers, over the same steps of
    # the scene as the headline arm (a fresh particle set, W untimed steps)
    e2e = None
    if not args.no_e2e:
        sim.close()
        sim = make_sim("warm" if warm is not None else "plain")
        for _ in range(args.warmup):
            sim.step(1)
        e2e = run_e2e(sim, args, dist, world, n)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            v, info = reference_sample(args.config, args.ref_iterations,
                                       target_s=args.ref_seconds, max_steps=40)
            cpu = {"value": v, "unit": UNIT, "cores": info["cores"], "kind": info["kind"],
                   "sample": info["sample"]}
        except Exception as e:  # the checker is optional on a box without it
            cpu = {"value": None, "unit": UNIT, "cores": 1, "kind": "reference",
                   "sample": f"unavailable: {e}"}
    sim.close()
    if rank != 0:
        return
    clocks = head["clocks"]
    like = None
    if fixed is not None:
        fv = job_rate(world, n, args.steps, fixed["ms"] / 1e3)
        like = {"iterations": args.ref_iterations, "gpu_value": fv,
                "gpu_ms_per_step": fixed["ms"] / args.steps,
                "reference_value": cpu["value"] if cpu else None,
                "ratio": (fv / cpu["value"]) if cpu and cpu.get("value") else None,
                "note": "both at the reference arm's fixed iteration count; the reference "
                        "runs a 32x32x32 block of the scene on one core"}

    def arm_summary(a):
        if a is None:
            return None
        return {"value": job_rate(world, n, args.steps, a["ms"] / 1e3),
                "ms_per_step": a["ms"] / args.steps,
                "mean_iterations": float(np.mean(a["iters"])) if a["iters"] else None,
                "steps_converged": a["converged"] if a["iters"] else None,
                "steps_unconverged": (len(a["iters"]) - a["converged"]) if a["iters"] else None,
                "warm_start_steps": a["warm_used"], "gate_rejections": a["rejected"],
                "final_max_density_error": a["diag"]["max_density_error"],
                "gpu_launches": a["launches"]}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
        "data": "synthetic",
        "config": {"workload": args.config, "particles_per_gpu": n,
                   "solver": ("fixed iterations" if args.fixed else
                              f"iterate to max density err <= {args.tol} (cap {args.max_iters}"
                              + (f"; stop when two iterations lower it by < "
                                 f"{100 * args.min_progress:g}%" if args.min_progress > 0 else "")
                              + ")")
                   + ((", MLP warm start (output scale "
                       f"{warm_settings['scale']:g}, network skipped at feature-pass error <= "
                       f"{warm_settings['min_error']:g}, residual gate "
                       f"{'on' if warm_settings['gate'] else 'off'})")
                      if warm is not None else ", plain (no network file)"),
                   "plain": arm_summary(plain),
                   "warm_start": arm_summary(warm),
                   "carried_multiplier_start": arm_summary(carry),
                   "warm_start_weights": (os.path.relpath(args.weights, ROOT)
                                          if warm is not None else None),
                   "speedup_vs_plain": (plain["ms"] / warm["ms"]) if warm is not None else None,
                   "speedup_carried_vs_plain": (plain["ms"] / carry["ms"])
                   if carry is not None else None,
                   "stiffness_k": args.stiffness_k,
                   "mean_iterations": float(np.mean(iters)) if iters else None,
                   "steps_converged": conv if iters else None,
                   "l2": "state larger than L2 (no flush)",
                   "final_max_density_error": diag["max_density_error"],
                   "parallelism": f"replicas x{world}"},
        "gpu_launches": launches,
        "clocks": clocks,
        "roofline": roof,
        "hbm_class_roofline": hbm_class,
        "neighbour_stage_roofline": nbr_stages,
        "stage_ms_per_step": {k: v[1] / args.steps for k, v in prof.items()},
        "like_for_like": like,
        "e2e": e2e,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


def sim_cells(sim):
    return sim.neighbors.hash_size_x * sim.neighbors.hash_size_y * sim.neighbors.hash_size_z


def sim_passes(sim):
    """Digit passes of the step's sort: 8-bit digits over the cell keys' bits."""
    C_ = sim_cells(sim)
    bits = max(1, int(C_ - 1).bit_length())
    return (bits + 7) // 8


def ncu_stage(stage):
    """The committed ncu figures of `stage` (profiles/ncu_traffic.json), or {}."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        with open(path) as f:
            return json.load(f).get(stage, {})
    except Exception:
        return {}


def ncu_traffic(stage, n):
    """DRAM bytes per launch of `stage` from the committed ncu summary, scaled
    to n particles, or None."""
    e = ncu_stage(stage)
    return e["bytes_per_particle"] * n if "bytes_per_particle" in e else None


def run_e2e(sim, args, dist, world, n):
    """Host buffers in, host buffers out, through the public C API: upload the
    state from the host arrays (x, v), K steps each followed by the FP64
    diagnostics read-back, the reference's output frame (x, y, z, density
    every 1/(30 dt) steps, simulation.c:113-114, read back asynchronously),
    and the final state."""
    import torch
    fields_in = ["x", "y", "z", "v_x", "v_y", "v_z"]
    frame_fields = ["x", "y", "z", "density"]
    out_fields = ["x", "y", "z", "v_x", "v_y", "v_z", "density"]
    frame_every = max(1, int(1.0 / (sim.params.time_step * 30.0)))
    sim.fetch_fields(fields_in)  # host arrays hold a valid state
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sim.push_fields(fields_in)
    frames = 0
    for k in range(args.steps):
        sim.step(1)
        sim.diagnostics()
        if k % frame_every == 0:
            # the frame crosses the link while the next steps run; the next
            # frame (or the final read-back) waits for it first
            sim.fetch_fields_async(frame_fields)
            frames += 1
    sim.host_wait()
    sim.fetch_fields(out_fields)
    torch.cuda.synchronize()
    dt = max_over_ranks(time.perf_counter() - t0, dist, "cuda")
    h2d = 8 * len(fields_in) * n
    d2h = args.steps * 72 + frames * 8 * len(frame_fields) * n + 8 * len(out_fields) * n
    return {"value": job_rate(world, n, args.steps, dt), "unit": UNIT,
            "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
            "host_memory": "the reference's calloc'd arrays, page-locked in place by the "
                           "library (cudaHostRegister at enter_data)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="full_16m")
    ap.add_argument("--tol", type=float, default=0.01)
    ap.add_argument("--max-iters", type=int, default=12)
    ap.add_argument("--min-progress", type=float, default=0.02,
                    help="adaptive solver: stop (step not converged) when two iterations "
                         "lower the max density error by less than this fraction; 0: off")
    ap.add_argument("--fixed", action="store_true", help="configured iteration count")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-warm", action="store_true", help="plain solver only")
    ap.add_argument("--arms", default="plain,warm,carry,fixed",
                    help="solver arms, each from the same initial state: plain, warm (the "
                         "network's multipliers), carry (the previous step's applied "
                         "multipliers carried through the sort, no network), fixed (the "
                         "reference arm's fixed iteration count, --ref-iterations)")
    ap.add_argument("--stiffness-k", type=float, default=None,
                    help="UpdateDPs stiffness constant k of s_n = 1 - (1 - k)^(1/n) "
                         "(the reference's 0.95 by default; 1 gives a constant 1)")
    ap.add_argument("--weights", default=os.path.join(ROOT, "sphpc_b200", "weights",
                                                      "warm_start.npz"))
    ap.add_argument("--warm-scale", type=float, default=None,
                    help="multiplier on the network's output (default: the one stored "
                         "with the network)")
    ap.add_argument("--warm-min-error", type=float, default=None,
                    help="first-pass max density error below which the network is skipped "
                         "(default: the one stored with the network)")
    ap.add_argument("--warm-gate", type=int, default=1,
                    help="1: discard a warm pass that does not lower the FP64 max density "
                         "error (the residual gate); 0: keep every warm pass")
    ap.add_argument("--ref-iterations", type=int, default=6)
    ap.add_argument("--ref-seconds", type=float, default=8.0)
    args = ap.parse_args()
    world, rank, local, dist = dist_init(args)
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_ours(args, world, rank, local, dist)
    finally:
        if dist:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
