"""Slab decomposition (sphpc_slab_*, sphpc_b200/slab.py) on one device: the
32,768-particle dam break split into three x-slabs held by one process, the
records handed over by device copies, against the undivided run.  Each slab
works on its own particles plus its neighbours' within the halo width, so
its own particles' positions and velocities must equal the undivided run's
bit for bit while the fluid flows across the slab ends (particles change
owner, over 200 steps); every particle is owned by exactly one slab.  A slab
narrower than the halo between two neighbours is refused."""
import numpy as np
import pytest

from sphpc_b200 import slab
from sphpc_b200.simulation import Simulation

pytestmark = pytest.mark.gpu

# the middle slab (both neighbours) is wider than the halo (21.6 here)
BOUNDS = [(0.0, 16.0), (16.0, 38.0), (38.0, 96.0)]


def _owned_union(domains):
    gs, xs, vs = [], [], []
    for d in domains:
        g, x, v = d.owned()
        gs.append(g)
        xs.append(x)
        vs.append(v)
    g = np.concatenate(gs)
    o = np.argsort(g, kind="stable")
    return g[o], np.concatenate(xs)[o], np.concatenate(vs)[o], [len(a) for a in gs]


def _owners(domains, n):
    owner = np.full(n, -1)
    for r, d in enumerate(domains):
        g, _, _ = d.owned()
        assert np.all(owner[g] == -1)
        owner[g] = r
    assert np.all(owner >= 0)
    return owner


def test_three_slabs_equal_the_undivided_run():
    steps_per_check = (1, 9, 190)
    with Simulation("dam_break_32k") as whole:
        n = whole.n
        sims = [Simulation("dam_break_32k") for _ in BOUNDS]
        try:
            domains = [slab.SlabDomain(s, lo, hi, k > 0, k < len(BOUNDS) - 1)
                       for k, (s, (lo, hi)) in enumerate(zip(sims, BOUNDS))]
            assert domains[0].width < 24.0   # the slabs see only part of the scene
            first_owner = None
            for k in steps_per_check:
                whole.step(k)
                slab.step_local(domains, k)
                g, x, v, counts = _owned_union(domains)
                np.testing.assert_array_equal(g, np.arange(n, dtype=np.uint32))
                st = whole.fetch(["x", "y", "z", "v_x", "v_y", "v_z"])
                want_x = np.stack([st["x"], st["y"], st["z"]], 1)
                want_v = np.stack([st["v_x"], st["v_y"], st["v_z"]], 1)
                np.testing.assert_array_equal(x, want_x)
                np.testing.assert_array_equal(v, want_v)
                if first_owner is None:
                    first_owner = _owners(domains, n)
            # the slab farthest from the initial block sees only part of the
            # scene (the middle slab's halo spans the whole early block)
            assert sims[2].particles.local_count < n
            # one more exchange hands every particle to the slab its position
            # lies in; the fluid crossed slab ends, so some changed owner
            slab.exchange_local(domains)
            owner = _owners(domains, n)
            st = whole.fetch(["x"])
            edges = np.array([b[0] for b in BOUNDS[1:]])
            np.testing.assert_array_equal(owner, np.searchsorted(edges, st["x"], side="right"))
            assert np.sum(owner != first_owner) > 0
            for s in sims:
                assert s.device_errors() == 0
        finally:
            for s in sims:
                s.close()


def test_slab_narrower_than_the_halo_is_refused():
    with Simulation("dam_break_32k") as sim:
        with pytest.raises(ValueError):
            slab.SlabDomain(sim, 16.0, 30.0, True, True)
