"""ctypes front end of the CPU oracle (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module, as the checker of the CUDA path.  PARITY UNPINNED (see
finflo_oracle.h).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from finflo_b200.case import FFPatch, FFParams, SLOTS

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def build(force=False):
    so = os.path.join(_HERE, "liboracle.so")
    src = os.path.join(_HERE, "finflo_oracle.c")
    if force or not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE, "liboracle.so", "CC=gcc"])
    return so


def lib():
    global _LIB
    if _LIB is None:
        _LIB = ctypes.CDLL(build())
        L = _LIB
        vp = ctypes.c_void_p
        for name in ("orc_statim", "orc_refcen", "orc_time3", "orc_predgs", "orc_diaggs",
                     "orc_corrgs", "orc_fin_limits", "orc_boundi"):
            getattr(L, name).restype = None
        L.orc_roe_face.restype = None
    return _LIB


class OrcBlock(ctypes.Structure):
    _fields_ = [("imax", ctypes.c_int), ("jmax", ctypes.c_int), ("kmax", ctypes.c_int),
                ("npatch", ctypes.c_int), ("patch", ctypes.POINTER(FFPatch)),
                ("a", ctypes.c_void_p * len(SLOTS))]


class Oracle:
    """Wraps one block's numpy arrays (modified in place by the oracle)."""

    def __init__(self, blk, prm: FFParams):
        self.blk = blk
        self.prm = prm
        self._patches = blk.patch_array()
        ob = OrcBlock()
        ob.imax, ob.jmax, ob.kmax = blk.imax, blk.jmax, blk.kmax
        ob.npatch = len(blk.patches)
        ob.patch = ctypes.cast(self._patches, ctypes.POINTER(FFPatch))
        for i, n in enumerate(SLOTS):
            arr = blk.arrays[n]
            assert arr.dtype == np.float64 and arr.flags.c_contiguous
            ob.a[i] = arr.ctypes.data
        self.ob = ob
        self.L = lib()

    def _b(self):
        return ctypes.byref(self.ob)

    def _p(self):
        return ctypes.byref(self.prm)

    def statim(self):
        self.L.orc_statim(self._b(), self._p())

    def boundi(self):
        self.L.orc_boundi(self._b(), self._p())

    def subin(self):
        d = ctypes.c_double()
        self.L.orc_subin(self._b(), ctypes.byref(d))
        return d.value

    def adjuin(self):
        self.L.orc_adjuin_laminar(self._b())

    def residu(self, level=1, icycle=1):
        self.L.orc_residu(self._b(), self._p(), level, icycle)

    def resl2(self):
        r = (ctypes.c_double * 5)()
        self.L.orc_resl2(self._b(), r)
        return np.array(r[:])

    def imps(self, level=1):
        self.L.orc_imps(self._b(), self._p(), level)

    def time3(self, cfl):
        self.L.orc_time3(self._b(), self._p(), ctypes.c_double(cfl))

    def locdt_copr(self):
        self.L.orc_locdt_copr(self._b())

    def predgs(self):
        self.L.orc_predgs(self._b(), self._p())

    def diaggs(self):
        self.L.orc_diaggs(self._b(), self._p())

    def corrgs(self):
        self.L.orc_corrgs(self._b(), self._p())

    def ddadi(self):
        self.L.orc_ddadi(self._b(), self._p())

    def time_levels(self, mode):
        """TIMEL: mode 0 = STARTI (both old levels = the state), 1 = NEWTIM."""
        self.L.orc_time_levels(self._b(), 7 if self.prm.iturb >= 3 else 5, mode)

    def fin_limits(self):
        self.L.orc_fin_limits(self._b(), self._p())

    def cycle(self, icycle):
        r = (ctypes.c_double * 5)()
        d = ctypes.c_double()
        fn = self.L.orc_cycle_sst if self.prm.iturb >= 3 else self.L.orc_cycle
        fn(self._b(), self._p(), icycle, r, ctypes.byref(d))
        return np.array(r[:]), d.value

    def turbeq(self):
        self.L.orc_turbeq_sst(self._b(), self._p())

    def residu_sst(self, icycle=1):
        self.L.orc_residu_sst(self._b(), self._p(), icycle)

    def imps_sst(self):
        self.L.orc_imps_sst(self._b(), self._p())

    def fin_limits_sst(self):
        self.L.orc_fin_limits_sst(self._b(), self._p())

    def start(self):
        """NS3D start-up: SUBIN(0), BOUNDI(1) (ns3c.f:378-379), then SUBIN copies."""
        self.subin()
        self.boundi()
        self.subin()
        if self.prm.iturb >= 3:
            a = self.blk.arrays
            a["RKOLD"][:] = a["RK"]
            a["EPSOLD"][:] = a["REPS"]


def roe_face(qr, ql, qrr, qll, nrm, area, intem, prm, cell_r, cell_l, kquirk=False):
    L = lib()
    D5 = ctypes.c_double * 5
    f = D5(0, 0, 0, 0, 0)
    L.orc_roe_face(D5(*qr), D5(*ql), D5(*qrr), D5(*qll), (ctypes.c_double * 3)(*nrm),
                   ctypes.c_double(area), intem, ctypes.byref(prm), D5(*cell_r), D5(*cell_l),
                   int(kquirk), f)
    return np.array(f[:])


class OracleMG:
    """Multigrid levels of one block (finest first) for orc_mg_cycle."""

    def __init__(self, levels, prms):
        self.levels = [Oracle(b, p) for b, p in zip(levels, prms)]
        n = len(levels)
        self._ptrs = (ctypes.POINTER(OrcBlock) * n)(*[ctypes.pointer(o.ob) for o in self.levels])
        self._prms = (FFParams * n)(*prms)
        self.L = lib()

    def start(self):
        self.levels[0].start()

    def cycle(self, icycle):
        r = (ctypes.c_double * 5)()
        d = ctypes.c_double()
        fn = self.L.orc_mg_cycle_sst if self._prms[0].iturb >= 3 else self.L.orc_mg_cycle
        fn(self._ptrs, len(self.levels), self._prms, icycle, r, ctypes.byref(d))
        return np.array(r[:]), d.value


class OracleMB:
    """Single-grid blocks joined by 1:1 patches, for orc_mb_cycle."""

    def __init__(self, blocks, prms):
        self.blocks = [Oracle(b, p) for b, p in zip(blocks, prms)]
        n = len(blocks)
        self._ptrs = (ctypes.POINTER(OrcBlock) * n)(*[ctypes.pointer(o.ob) for o in self.blocks])
        self._prms = (FFParams * n)(*prms)
        self.L = lib()

    def boundi(self):
        self.L.orc_mb_boundi(self._ptrs, len(self.blocks), self._prms)

    def start(self):
        """NS3D start-up over all blocks: SUBIN, BOUNDI(1), SUBIN."""
        for o in self.blocks:
            o.subin()
        self.boundi()
        for o in self.blocks:
            o.subin()

    def cycle(self, icycle):
        r = (ctypes.c_double * 5)()
        d = ctypes.c_double()
        self.L.orc_mb_cycle(self._ptrs, len(self.blocks), self._prms, icycle, r, ctypes.byref(d))
        return np.array(r[:]), d.value


class OracleMBMG:
    """Blocks joined by 1:1 patches, each with its multigrid levels (finest
    first), for orc_mb_mg_cycle.  A 1:1 patch's IBTYPE is the source block's
    index in block_levels."""

    def __init__(self, block_levels, block_prms):
        self.nblk, self.nlev = len(block_levels), len(block_levels[0])
        self.objs = [[Oracle(b, p) for b, p in zip(lv, pr)] for lv, pr in zip(block_levels, block_prms)]
        flat = [o for lv in self.objs for o in lv]
        self._ptrs = (ctypes.POINTER(OrcBlock) * len(flat))(*[ctypes.pointer(o.ob) for o in flat])
        self._prms = (FFParams * len(flat))(*[p for pr in block_prms for p in pr])
        self.fine = OracleMB([lv[0] for lv in block_levels], [pr[0] for pr in block_prms])
        self.L = lib()

    def start(self):
        """NS3D start-up over the level-1 blocks: SUBIN, BOUNDI(1), SUBIN (and
        the k-omega *OLD copies)."""
        self.fine.start()
        for lv in self.objs:
            o = lv[0]
            if o.prm.iturb >= 3:
                a = o.blk.arrays
                a["RKOLD"][:] = a["RK"]
                a["EPSOLD"][:] = a["REPS"]

    def cycle(self, icycle):
        r = (ctypes.c_double * 5)()
        d = ctypes.c_double()
        self.L.orc_mb_mg_cycle(self._ptrs, self.nblk, self.nlev, self._prms, icycle, r, ctypes.byref(d))
        return np.array(r[:]), d.value
