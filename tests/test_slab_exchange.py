"""The slab decomposition's neighbour exchange (sphpc_b200/slab.py,
DistExchange) over torch.distributed with gloo on the CPU: 2 and 3 ranks in
slab order, each sending distinct records to its left and right neighbours
(counts first, then the records, as the reference's ExchangeHalo /
ExchangeOOB trade them with MPI, communication.c:222-585); every rank must
receive exactly its neighbours' records, and the end ranks none from beyond.
No GPU: the records are host buffers."""
import os
import socket

import numpy as np
import pytest


def _records(rank, side, n):
    """n 32-byte records from `rank` towards `side` (0 left, 1 right)."""
    a = np.zeros((n, 8), np.uint32)
    a[:, 3] = rank * 1000 + side * 500 + np.arange(n)
    a[:, 7] = side
    return a.view(np.uint8).reshape(-1)


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from sphpc_b200.slab import DistExchange
        ex = DistExchange(rank, world, device="cpu")
        out = []
        for step in range(3):
            nl, nr = 3 + rank + step, 5 + 2 * rank
            sl = torch.from_numpy(_records(rank, 0, nl).copy())
            sr = torch.from_numpy(_records(rank, 1, nr).copy())
            rl, nfl, rr, nfr = ex.exchange(sl, nl if rank > 0 else 0, sr,
                                           nr if rank < world - 1 else 0)
            out.append((nfl, rl[:nfl * 32].numpy().copy(), nfr, rr[:nfr * 32].numpy().copy()))
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
def test_neighbour_exchange_gloo(world):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank in range(world):
        for step, (nfl, rl, nfr, rr) in enumerate(results[rank]):
            if rank > 0:   # the left neighbour's records sent to its right
                nr = 5 + 2 * (rank - 1)
                assert nfl == nr
                np.testing.assert_array_equal(rl, _records(rank - 1, 1, nr))
            else:
                assert nfl == 0
            if rank < world - 1:   # the right neighbour's records sent to its left
                nl = 3 + (rank + 1) + step
                assert nfr == nl
                np.testing.assert_array_equal(rr, _records(rank + 1, 0, nl))
            else:
                assert nfr == 0
