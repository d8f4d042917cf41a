"""Oracle-backed compute for the multi-rank driver (test infrastructure).

Implements the device phases of ``finflo_b200.dist`` with the CPU oracle so
that the partition, the halo plan and the send/recv exchange can be run as
gloo ranks on CPU and compared with the single-process oracle.
"""
import ctypes

import numpy as np
import torch

from finflo_b200 import dist as fd
from finflo_b200 import grid
from oracle.oracle import Oracle, lib


class OracleBackend:
    device = torch.device("cpu")

    def add_blocks(self, blocks, prms):
        self.blocks = blocks
        self.orcs = [Oracle(b, p) for b, p in zip(blocks, prms)]
        self.hist = []
        self.resi = np.zeros(5)

    def set_halo(self, items, send, recv):
        self.items, self.send, self.recv = list(items), send, recv

    def _buf(self, t, off):
        return ctypes.c_void_p(t.data_ptr() + 8 * off)

    def phase(self, phase, icycle, use_graph=True):
        L = lib()
        if phase == fd.PHASE_CYCLE_A:
            self.resi = np.zeros(5)
            for o in self.orcs:
                o.statim(); o.adjuin(); o.residu(1, icycle)
                self.resi += o.resl2()
                o.imps(1); o.fin_limits()
        if phase in (fd.PHASE_CYCLE_A, fd.PHASE_BOUNDI_A):
            for o in self.orcs:
                L.orc_refcor(o._b()); L.orc_mir(o._b()); o.statim()
            for o in self.orcs:
                for ip in range(o.ob.npatch):
                    pa = o._patches[ip]
                    if pa.ityp == grid.BC_CON and pa.ibtype >= 0:
                        L.orc_connec_patch(o._b(), ctypes.byref(pa), ctypes.byref(self.orcs[pa.ibtype].ob))
            for it in self.items:
                if it.mode == 0:
                    L.orc_halo_pack(ctypes.byref(self.orcs[it.blk].ob), ctypes.byref(it.pa),
                                    self._buf(self.send, it.offset))
        elif phase == fd.PHASE_B:
            for it in self.items:
                if it.mode == 1:
                    L.orc_halo_unpack(ctypes.byref(self.orcs[it.blk].ob), ctypes.byref(it.pa),
                                      self._buf(self.recv, it.offset))
            for o in self.orcs:
                o.statim()
        elif phase == fd.PHASE_RECORD:
            dm = max(o.subin() for o in self.orcs)
            self.hist.append(list(self.resi) + [dm])

    def exchange_stream(self):
        import contextlib
        return contextlib.nullcontext()

    def sync(self):
        pass

    def start_copies(self):
        for o in self.orcs:
            o.subin()

    def reserve_history(self, n):
        self.hist = []

    def history(self, n):
        return np.array(self.hist[:n])
