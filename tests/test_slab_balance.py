"""BalanceNodes (geometry.c:102-166) through the C ABI (sphpc_balance_nodes)
against a restatement of the reference's rule, and the halo width the
one-exchange-per-step decomposition needs (no GPU)."""
import ctypes as C

import numpy as np

from sphpc_b200 import _lib
from sphpc_b200._lib import Params, Solver
from sphpc_b200.slab import balance_nodes


def _reference_rule(rank, procs, num_rank, num_right, start, end, ll, lr, global_count, h):
    """geometry.c:102-166 restated (the C int / float conversions included)."""
    length = end - start
    even = int(global_count / float(procs))
    max_diff = int(np.float32(even) / np.float32(10.0))
    diff_right = num_right - even
    diff_self = num_rank - even
    if diff_self > max_diff and length > 2 * h and rank != 0:
        start += h
    elif diff_self < -max_diff and ll > 2 * h and rank != 0:
        start -= h
    if diff_right > max_diff and lr > 2 * h and rank != procs - 1:
        end += h
    elif diff_right < -max_diff and length > 2 * h and rank != procs - 1:
        end -= h
    return start, end


def test_balance_nodes_matches_the_reference_rule():
    rng = np.random.default_rng(3)
    h = 2.0
    for _ in range(300):
        procs = int(rng.integers(1, 9))
        edges = np.sort(rng.uniform(0, 400, procs - 1)) if procs > 1 else np.array([])
        edges = np.concatenate([[0.0], edges, [400.0]])
        bounds = [(float(edges[r]), float(edges[r + 1])) for r in range(procs)]
        counts = [int(c) for c in rng.integers(0, 20000, procs)]
        total = int(sum(counts))
        got = balance_nodes(procs, counts, bounds, total, h)
        for r in range(procs):
            ll = bounds[r - 1][1] - bounds[r - 1][0] if r > 0 else 0.0
            lr = bounds[r + 1][1] - bounds[r + 1][0] if r + 1 < procs else 0.0
            nr = counts[r + 1] if r + 1 < procs else 0
            want = _reference_rule(r, procs, counts[r], nr, bounds[r][0], bounds[r][1], ll, lr,
                                   total, h)
            assert got[r] == want, (r, got[r], want)


def test_balance_nodes_moves_towards_an_even_share():
    # rank 1 holds far more than its share: its start moves right, rank 0's
    # end follows
    out = balance_nodes(3, [100, 1000, 100], [(0, 100), (100, 200), (200, 300)], 1200, 2.0)
    assert out[1][0] == 102.0 and out[0][1] == 102.0


def test_halo_width_covers_every_neighbour_hop():
    p = Params()
    p.smoothing_radius = 2.0
    p.time_step = 0.008
    s = Solver()
    _lib.load().sphpc_default_solver(C.byref(s))
    s.solve_iterations = 6
    s.surface_tension = 1
    s.vorticity = 1
    s.velocity_max = 100.0
    w = C.c_double()
    _lib.call("sphpc_slab_halo_width", C.byref(p), C.byref(s), C.byref(w))
    hops = 2 * 6 + 2 + 1 + 2
    assert w.value == (hops + 1) * 2.0 + 2 * 100.0 * 0.008
