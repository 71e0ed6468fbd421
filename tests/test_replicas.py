"""bench.py's multi-GPU host logic (replicas only: barriers and the
max-over-ranks time are the only collectives) with two gloo ranks on CPU."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port),
                       "WORLD_SIZE": str(world), "RANK": str(rank), "LOCAL_RANK": str(rank)})
    sys.path.insert(0, ROOT)
    import bench
    w, r, local, dist = bench.dist_init(None, backend="gloo")
    try:
        dist.barrier()
        # rank r "took" (r + 1) * 10 ms: the job's time is the slowest rank's
        ms = bench.max_over_ranks((r + 1) * 10.0, dist, "cpu")
        q.put((r, w, ms, bench.job_rate(w, 1000, 5, ms / 1e3)))
    finally:
        dist.destroy_process_group()


def test_two_replicas_time_is_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, w, ms, rate in got:
        assert w == 2 and ms == pytest.approx(20.0)
        # 2 replicas x 1000 particles x 5 steps in 20 ms
        assert rate == pytest.approx(2 * 1000 * 5 / 0.020)


def test_reference_arm_prints_on_rank_zero_only(capsys):
    sys.path.insert(0, ROOT)
    import bench

    class A:
        config = "dam_break_32k"
        ref_iterations = 1
        warmup = 0
        steps = 1
    bench.run_reference(A, 2, 1)   # a non-zero rank exits without work
    assert capsys.readouterr().out == ""


def test_reference_arm_line_keeps_the_bench_contract(capsys):
    """`bench.py --impl reference` on rank 0: one JSON line with the bench
    contract's keys, the reference arm's marker and its CPU baseline, e2e
    without host-device copies (a one-step, one-iteration sample)."""
    import json

    sys.path.insert(0, ROOT)
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libsphpc_ref_fast.so")):
        pytest.skip("the reference's CPU path is not built here")
    import bench

    class A:
        config = "dam_break_32k"
        ref_iterations = 1
        warmup = 0
        steps = 1
    bench.run_reference(A, 1, 0)
    out = [l for l in capsys.readouterr().out.splitlines() if l.startswith("{")]
    assert len(out) == 1
    d = json.loads(out[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["n_gpus"] == 1
    assert d["metric"] == bench.METRIC and d["unit"] == bench.UNIT
    assert d["higher_is_better"] is True and d["steps"] == 1 and d["warmup"] == 0
    assert d["config"]["workload"] == "dam_break_32k"
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] == 1 and cb["value"] == d["value"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["h2d_bytes_per_step"] == 0
    assert e["d2h_bytes_per_step"] == 0
