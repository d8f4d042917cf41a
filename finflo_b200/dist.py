"""Blocks spread over several GPUs, one process per GPU.

The reference distributes whole blocks over MPI processes and swaps the
ghost layers of 1:1 patches between them every BOUNDI (EXPTOT / IMPVO2,
gluebm.f:6819 / 6964, called from CONNEC ns3c.f:8605); residual norms are
summed over processes for the convergence monitor.  Here:

* ``partition`` assigns blocks to ranks (largest first onto the least
  loaded rank), so each GPU holds whole blocks in its HBM;
* ``HaloPlan`` lists, per peer rank, the remote patches in one canonical
  order that both sides derive from the global block list, with the offsets
  of their packed ghost data ([layer][var][cell], 24 doubles per patch cell);
* ``DistributedBlocks`` drives one cycle as: device phase A (CYCLES of the
  local blocks, BOUNDI part one, local CONNEC, halo pack) -> one grouped
  send/recv per peer (NCCL over NVLink, or gloo on CPU) -> phase B (unpack,
  second STATIM) -> history row.  The per-cycle residual sums and max|dp|
  stay on each GPU and are reduced over ranks once, when the history is
  read, so the only per-cycle collective is the halo exchange itself.

The compute side is a backend object (``GpuBackend`` here: one
``GpuSolver`` context per GPU); the exchange and the plan are independent
of it.
"""
from __future__ import annotations

import contextlib
from dataclasses import dataclass

import numpy as np

from .case import Block, FFHaloItem, FFPatch
from . import grid

PHASE_CYCLE_A, PHASE_BOUNDI_A, PHASE_B, PHASE_RECORD = 0, 1, 2, 3
HALO_VARS = 12
HALO_LAYERS = 2


def partition(cells, world):
    """Owner rank of each block: largest blocks first, each onto the rank
    with the fewest cells so far (ties to the lower rank)."""
    load = [0] * world
    owner = [0] * len(cells)
    for b in sorted(range(len(cells)), key=lambda i: (-cells[i], i)):
        r = min(range(world), key=lambda q: (load[q], q))
        owner[b] = r
        load[r] += cells[b]
    return owner


def _copy_patch(pa):
    return FFPatch.from_buffer_copy(pa)


@dataclass
class Link:
    dst: int          # global id of the block whose ghosts are filled
    ip: int           # patch index in that block
    src: int          # global id of the source block
    pa: FFPatch       # the destination's patch
    n: int            # patch cells

    @property
    def doubles(self):
        return HALO_LAYERS * HALO_VARS * self.n


def links(blocks):
    out = []
    for d, b in enumerate(blocks):
        for ip, pa in enumerate(b.patches):
            if pa.ityp == grid.BC_CON:
                n = (pa.r1b - pa.r1a + 1) * (pa.r2b - pa.r2a + 1)
                out.append(Link(d, ip, pa.ibtype, pa, n))
    return out


class HaloPlan:
    """Local blocks, rewritten patch tables and the packed exchange of one
    rank."""

    def __init__(self, blocks, owner, rank):
        self.rank = rank
        self.local = [g for g in range(len(blocks)) if owner[g] == rank]
        self.lid = {g: i for i, g in enumerate(self.local)}
        # patch tables as the rank's context sees them: local sources by
        # local id, remote sources marked with a negative id
        self.patches = []
        for g in self.local:
            pats = []
            for pa in blocks[g].patches:
                q = _copy_patch(pa)
                if pa.ityp == grid.BC_CON:
                    q.ibtype = self.lid[pa.ibtype] if owner[pa.ibtype] == rank else -1 - pa.ibtype
                pats.append(q)
            self.patches.append(pats)
        remote = [l for l in links(blocks) if owner[l.src] != owner[l.dst]]
        key = lambda l: (l.dst, l.ip)
        self.items = []
        self.send_ranges, self.recv_ranges = {}, {}
        off = 0
        for q in sorted({owner[l.dst] for l in remote if owner[l.src] == rank}):
            start = off
            for l in sorted((l for l in remote if owner[l.src] == rank and owner[l.dst] == q), key=key):
                self.items.append(self._item(self.lid[l.src], 0, off, l.pa))
                off += l.doubles
            self.send_ranges[q] = (start, off - start)
        self.nsend = off
        off = 0
        for p in sorted({owner[l.src] for l in remote if owner[l.dst] == rank}):
            start = off
            for l in sorted((l for l in remote if owner[l.dst] == rank and owner[l.src] == p), key=key):
                self.items.append(self._item(self.lid[l.dst], 1, off, l.pa))
                off += l.doubles
            self.recv_ranges[p] = (start, off - start)
        self.nrecv = off

    @staticmethod
    def _item(blk, mode, off, pa):
        it = FFHaloItem()
        it.blk, it.mode, it.offset = blk, mode, off
        it.pa = _copy_patch(pa)
        return it

    def local_blocks(self, blocks):
        return [Block(blocks[g].imax, blocks[g].jmax, blocks[g].kmax, blocks[g].arrays, pats, blocks[g].nodes)
                for g, pats in zip(self.local, self.patches)]


class GpuBackend:
    """One GpuSolver context on this rank's GPU."""

    def __init__(self, device=0):
        import torch
        from .gpu import GpuSolver
        self.torch = torch
        self.device = torch.device("cuda", device)
        self.solver = GpuSolver(device)

    def add_blocks(self, blocks, prms):
        for b, p in zip(blocks, prms):
            bid = self.solver.add_block(b, p)
            self.solver.upload(bid)

    def set_halo(self, items, send, recv):
        self.solver.halo_plan(items, send.data_ptr() if send.numel() else 0,
                              recv.data_ptr() if recv.numel() else 0)

    def phase(self, phase, icycle, use_graph=True):
        self.solver.mb_phase(phase, icycle, use_graph)

    @contextlib.contextmanager
    def exchange_stream(self):
        s = self.torch.cuda.ExternalStream(self.solver.stream_handle(), device=self.device)
        with self.torch.cuda.stream(s):
            yield

    def sync(self):
        self.solver.sync()

    def start_copies(self):
        for bid in range(len(self.solver.blocks)):
            self.solver._old_copies(bid)

    def reserve_history(self, n):
        self.solver.reserve_history(n, reset=True)

    def history(self, n):
        return self.solver.history(n)

    def download(self, lid, names):
        return self.solver.download(lid, names)

    def close(self):
        self.solver.close()


class DistributedBlocks:
    """The blocks of a case spread over the ranks of a process group."""

    def __init__(self, blocks, prms, backend, group=None, owner=None):
        import torch
        import torch.distributed as dist
        self.torch, self.dist, self.group = torch, dist, group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.owner = owner or partition([b.interior_cells for b in blocks], self.world)
        self.plan = HaloPlan(blocks, self.owner, self.rank)
        self.backend = backend
        self.blocks = self.plan.local_blocks(blocks)
        backend.add_blocks(self.blocks, [prms[g] for g in self.plan.local])
        dev = backend.device
        self.send = torch.zeros(max(self.plan.nsend, 1), dtype=torch.float64, device=dev)
        self.recv = torch.zeros(max(self.plan.nrecv, 1), dtype=torch.float64, device=dev)
        backend.set_halo(self.plan.items, self.send[:self.plan.nsend], self.recv[:self.plan.nrecv])
        # every rank joins this first collective (NCCL wants all ranks in the
        # first one); it also checks that the plans agree
        tot = torch.tensor([self.plan.nsend, self.plan.nrecv], dtype=torch.float64, device=dev)
        dist.all_reduce(tot, group=group)
        if tot[0].item() != tot[1].item():
            raise RuntimeError("halo plans of the ranks disagree")

    def exchange(self):
        dist = self.dist
        ops = []
        for q, (o, n) in self.plan.send_ranges.items():
            ops.append(dist.P2POp(dist.isend, self.send[o:o + n], q, self.group))
        for p, (o, n) in self.plan.recv_ranges.items():
            ops.append(dist.P2POp(dist.irecv, self.recv[o:o + n], p, self.group))
        if not ops:
            return
        with self.backend.exchange_stream():
            for r in dist.batch_isend_irecv(ops):
                r.wait()

    def boundi(self):
        self.backend.phase(PHASE_BOUNDI_A, 1, False)
        self.exchange()
        self.backend.phase(PHASE_B, 1, False)

    def start(self):
        """NS3D start-up: BOUNDI(1) over all blocks, then the *OLD copies."""
        self.boundi()
        self.backend.sync()
        self.backend.start_copies()

    def cycles(self, n, icycle0=1, use_graph=True):
        """n cycles; returns the history over all ranks (sums of squares
        summed, max|dp| maximised)."""
        b = self.backend
        b.reserve_history(n)
        for i in range(n):
            ic = icycle0 + i
            b.phase(PHASE_CYCLE_A, ic, use_graph)
            self.exchange()
            b.phase(PHASE_B, ic, use_graph)
            b.phase(PHASE_RECORD, ic, use_graph)
        return self.reduce_history(b.history(n))

    def reduce_history(self, h):
        torch, dist = self.torch, self.dist
        t = torch.as_tensor(np.ascontiguousarray(h), dtype=torch.float64).to(self.backend.device)
        s = t[:, :5].contiguous()
        m = t[:, 5].contiguous()
        dist.all_reduce(s, op=dist.ReduceOp.SUM, group=self.group)
        dist.all_reduce(m, op=dist.ReduceOp.MAX, group=self.group)
        return np.concatenate([s.cpu().numpy(), m.cpu().numpy()[:, None]], axis=1)
