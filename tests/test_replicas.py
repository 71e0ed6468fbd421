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
