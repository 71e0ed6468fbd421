"""Slab decomposition of a scene along x over ranks, one GPU each (the
reference's Simulation/src/communication.c and BalanceNodes,
geometry.c:102-166), driven through the C ABI (include/sphpc.h,
sphpc_slab_*).

Every step is one exchange with each neighbour, then the fused step:

    pack (device)  -> records for the left / right neighbour, the rest kept
    exchange       -> record counts, then the records (device memory)
    unpack (device)-> working set = own particles + neighbours' halo copies
    sphpc_step     -> the owned particles' results equal the undivided run

The exchange is a transport object with
``exchange(send_left, n_left, send_right, n_right) -> (recv_left, n_from_left,
recv_right, n_from_right)`` over 32-byte records:

* ``DistExchange``: torch.distributed point-to-point with the neighbouring
  ranks (NCCL on device buffers over NVLink; gloo on host buffers);
* ``step_local``: several slabs held by one process (one device), the
  records handed over by device copies.
"""
from __future__ import annotations

import ctypes as C

from ._lib import Solver, call

RECORD_BYTES = 32


def halo_width(sim) -> float:
    """Halo width one exchange per step needs for the set's solver."""
    w = C.c_double()
    s = Solver()
    call("sphpc_get_solver", C.byref(sim.particles), C.byref(s))
    call("sphpc_slab_halo_width", C.byref(sim.params), C.byref(s), C.byref(w))
    return w.value


class SlabDomain:
    """One slab [node_start, node_end) of a decomposed scene, held by `sim`
    (a Simulation on this rank's device).  The scene may be loaded whole on
    every rank: the particles outside the slab leave at the first pack."""

    def __init__(self, sim, node_start: float, node_end: float, has_left: bool,
                 has_right: bool, send_capacity: int | None = None):
        import torch
        self.sim = sim
        self.node_start, self.node_end = float(node_start), float(node_end)
        self.has_left, self.has_right = bool(has_left), bool(has_right)
        sim.params.node_start_x = self.node_start
        sim.params.node_end_x = self.node_end
        solver = Solver()
        call("sphpc_get_solver", C.byref(sim.particles), C.byref(solver))
        if solver.adaptive or solver.warm_start:
            sim.set_solver(adaptive=0, warm_start=0)
        self.width = halo_width(sim)
        # halo copies come from the two neighbours only: a slab between two
        # neighbours must hold every particle its neighbours' halos need
        if self.has_left and self.has_right and self.node_end - self.node_start < self.width:
            raise ValueError(f"slab [{self.node_start}, {self.node_end}) is narrower than the "
                             f"halo width {self.width:.3g} (its neighbours would need particles "
                             f"two slabs away)")
        call("sphpc_slab_init", C.byref(sim.particles), 0, self.node_start, self.node_end,
             int(self.has_left), int(self.has_right))
        cap = send_capacity or max(1024, sim.particles.max_local // 2)
        self.capacity = int(cap)
        dev = torch.device("cuda", torch.cuda.current_device())
        self.send = [torch.empty(self.capacity * RECORD_BYTES, dtype=torch.uint8, device=dev)
                     for _ in range(2)]
        self.recv = [torch.empty(self.capacity * RECORD_BYTES, dtype=torch.uint8, device=dev)
                     for _ in range(2)]

    def pack(self):
        """Records for the neighbours; returns (n_left, n_right)."""
        nl, nr = C.c_int(), C.c_int()
        call("sphpc_slab_pack", C.byref(self.sim.particles), self.node_start, self.node_end,
             self.width, int(self.has_left), int(self.has_right),
             C.c_void_p(self.send[0].data_ptr()), C.c_void_p(self.send[1].data_ptr()),
             self.capacity, C.byref(nl), C.byref(nr))
        return nl.value, nr.value

    def unpack(self, recv_left, n_left, recv_right, n_right):
        call("sphpc_slab_unpack", C.byref(self.sim.particles),
             C.c_void_p(recv_left.data_ptr() if n_left else 0), int(n_left),
             C.c_void_p(recv_right.data_ptr() if n_right else 0), int(n_right))

    def owned(self):
        """(gids, positions [n, 3], velocities [n, 3]) of the owned particles,
        in global-id order."""
        import numpy as np
        cap = self.sim.particles.local_count
        g = np.empty(cap, np.uint32)
        x = np.empty(3 * cap, np.float64)
        v = np.empty(3 * cap, np.float64)
        n = C.c_int()
        call("sphpc_slab_owned", C.byref(self.sim.particles),
             g.ctypes.data_as(C.POINTER(C.c_uint)), x.ctypes.data_as(C.POINTER(C.c_double)),
             v.ctypes.data_as(C.POINTER(C.c_double)), cap, C.byref(n))
        k = n.value
        o = np.argsort(g[:k], kind="stable")
        return g[:k][o], x[:3 * k].reshape(-1, 3)[o], v[:3 * k].reshape(-1, 3)[o]

    def step(self, transport, steps: int = 1):
        """`steps` steps, each one exchange through `transport` and one fused
        step."""
        for _ in range(steps):
            nl, nr = self.pack()
            rl, nfl, rr, nfr = transport.exchange(self.send[0], nl, self.send[1], nr)
            self.unpack(rl, nfl, rr, nfr)
            self.sim.step(1)


class DistExchange:
    """Neighbour exchange of record buffers over torch.distributed (ranks in
    slab order along x).  Counts go first, then the records; every rank
    takes the same steps in the same order.  `device` is where the buffers
    live: the GPU for NCCL, "cpu" for gloo."""

    def __init__(self, rank: int, world: int, device="cuda", group=None):
        self.rank, self.world, self.device, self.group = rank, world, device, group
        self.left = rank - 1 if rank > 0 else None
        self.right = rank + 1 if rank < world - 1 else None
        self._recv = [None, None]

    def _p2p(self, sends, recvs):
        import torch.distributed as dist
        ops = [dist.P2POp(dist.isend, t, peer, self.group) for t, peer in sends] + \
              [dist.P2POp(dist.irecv, t, peer, self.group) for t, peer in recvs]
        if ops:
            for r in dist.batch_isend_irecv(ops):
                r.wait()

    def exchange(self, send_left, n_left, send_right, n_right):
        import torch
        dev = self.device
        cl = torch.tensor([n_left], dtype=torch.int64, device=dev)
        cr = torch.tensor([n_right], dtype=torch.int64, device=dev)
        fl = torch.zeros(1, dtype=torch.int64, device=dev)
        fr = torch.zeros(1, dtype=torch.int64, device=dev)
        sends, recvs = [], []
        if self.left is not None:
            sends.append((cl, self.left))
            recvs.append((fl, self.left))
        if self.right is not None:
            sends.append((cr, self.right))
            recvs.append((fr, self.right))
        self._p2p(sends, recvs)
        nfl, nfr = int(fl.item()), int(fr.item())
        for k, m in ((0, nfl), (1, nfr)):
            need = max(m, 1) * RECORD_BYTES
            if self._recv[k] is None or self._recv[k].numel() < need:
                self._recv[k] = torch.empty(need, dtype=torch.uint8, device=dev)
        sends, recvs = [], []
        if self.left is not None:
            if n_left:
                sends.append((send_left[:n_left * RECORD_BYTES], self.left))
            if nfl:
                recvs.append((self._recv[0][:nfl * RECORD_BYTES], self.left))
        if self.right is not None:
            if n_right:
                sends.append((send_right[:n_right * RECORD_BYTES], self.right))
            if nfr:
                recvs.append((self._recv[1][:nfr * RECORD_BYTES], self.right))
        self._p2p(sends, recvs)
        return self._recv[0], nfl, self._recv[1], nfr


def exchange_local(domains):
    """One exchange among slabs that one process holds (in slab order along
    x), the records handed over by device copies: afterwards every slab
    owns the particles whose positions lie in it, and holds its halo."""
    import torch
    counts = [d.pack() for d in domains]
    recv = []
    for i, d in enumerate(domains):
        nfl = counts[i - 1][1] if i > 0 else 0
        nfr = counts[i + 1][0] if i + 1 < len(domains) else 0
        if nfl:
            d.recv[0][:nfl * RECORD_BYTES].copy_(domains[i - 1].send[1][:nfl * RECORD_BYTES])
        if nfr:
            d.recv[1][:nfr * RECORD_BYTES].copy_(domains[i + 1].send[0][:nfr * RECORD_BYTES])
        recv.append((d.recv[0], nfl, d.recv[1], nfr))
    torch.cuda.synchronize()
    for d, r in zip(domains, recv):
        d.unpack(*r)


def step_local(domains, steps: int = 1):
    """Steps slabs that one process holds (in slab order along x): each step
    one exchange (exchange_local), then the fused step of every slab."""
    for _ in range(steps):
        exchange_local(domains)
        for d in domains:
            d.sim.step(1)


def balance_nodes(world: int, counts, bounds, global_count: int, h: float):
    """BalanceNodes (geometry.c:102-166) for every rank at once, given every
    rank's particle count and slab bounds: the new bounds."""
    from ._lib import Params
    out = []
    for r in range(world):
        p = Params()
        p.smoothing_radius = h
        p.node_start_x, p.node_end_x = bounds[r]
        ll = bounds[r - 1][1] - bounds[r - 1][0] if r > 0 else 0.0
        lr = bounds[r + 1][1] - bounds[r + 1][0] if r + 1 < world else 0.0
        nr = counts[r + 1] if r + 1 < world else 0
        call("sphpc_balance_nodes", r, world, int(counts[r]), int(nr), ll, lr, int(global_count),
             C.byref(p))
        out.append((p.node_start_x, p.node_end_x))
    return out
