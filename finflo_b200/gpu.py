"""Python front end of libfinflo_gpu.so (ctypes over the C-ABI of
include/finflo_gpu.h).

This is the host-side mirror of the reference's block-routine interface: a
``GpuSolver`` owns one device context and exposes the stage calls STATIM,
RESIDU, RESL2, IMPS, FIN, BOUNDI (ns3c.f:10318, 2355, res3c.f:8920,
ns3c.f:2683, res3c.f:1077, ns3c.f:10608) and the fused cycle loop of NS3D /
CYCLES (ns3c.f:467-663).  There is no CPU fallback: if the CUDA library is
missing or a device call fails, an exception is raised.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from .case import FFHaloItem, FFPatch, FFParams, SLOT, SLOTS, Block

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfinflo_gpu.so")
_SRC = [os.path.join(_HERE, "csrc", f) for f in ("ff_gpu.cu", "ff_kernels.cuh", "ff_device.cuh",
                                                 "ff_noalloc.cu", "ff_sst.cuh", "ff_pipe.cuh",
                                                 "ff_ddadi.cuh", "ff_grid.cuh", "ff_fortran.cu", "ff_fluxes.cuh")]
NVCC_FLAGS = ["-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
              "-Xcompiler", "-fPIC", "-shared", "-std=c++17"]

FF_STAGE_RESIDUAL, FF_STAGE_GRAD, FF_STAGE_STATE, FF_STAGE_SWEEP = 1, 2, 3, 4
FF_PHASE_CYCLE_A, FF_PHASE_BOUNDI_A, FF_PHASE_B, FF_PHASE_RECORD = 0, 1, 2, 3


class FinfloGpuError(RuntimeError):
    pass


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile libfinflo_gpu.so in-tree for sm_100a (nvcc cross-compiles
    without a GPU)."""
    newest = max(os.path.getmtime(p) for p in _SRC + [os.path.join(_HERE, "..", "include", "finflo_gpu.h"),
                                                      os.path.join(_HERE, "..", "include", "finflo_types.h")])
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < newest:
        cmd = ["nvcc"] + NVCC_FLAGS + ["-o", LIB_PATH, _SRC[0]]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd, cwd=os.path.join(_HERE, "csrc"))
    return LIB_PATH


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise FinfloGpuError(f"{LIB_PATH} is missing: run __graft_entry__.build() first")
        L = ctypes.CDLL(LIB_PATH)
        vp, ci, cd = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        L.ff_last_error.restype = ctypes.c_char_p
        L.ff_last_error.argtypes = [vp]
        L.ff_create.argtypes = [ctypes.POINTER(vp), ci]
        L.ff_destroy.argtypes = [vp]
        L.ff_block_add.argtypes = [vp, ci, ci, ci, ci, ctypes.POINTER(FFPatch), ctypes.POINTER(FFParams)]
        L.ff_block_params.argtypes = [vp, ci, ctypes.POINTER(FFParams)]
        L.ff_mg_link.argtypes = [vp, ci, ci]
        L.ff_boundi_all.argtypes = [vp]
        L.ff_halo_plan.argtypes = [vp, ci, ctypes.POINTER(FFHaloItem), vp, vp]
        L.ff_mb_phase.argtypes = [vp, ci, ci, ci]
        L.ff_history.argtypes = [vp, ci, ctypes.POINTER(cd), ci]
        L.ff_cycles_all.argtypes = [vp, ci, ci, ctypes.POINTER(cd), ci]
        L.ff_time_cycles_all.argtypes = [vp, ci, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ci)]
        L.ff_upload.argtypes = [vp, ci, ci, ctypes.POINTER(cd)]
        L.ff_download.argtypes = [vp, ci, ci, ctypes.POINTER(cd)]
        L.ff_device_ptr.restype = vp
        L.ff_device_ptr.argtypes = [vp, ci, ci]
        L.ff_stream.restype = vp
        L.ff_stream.argtypes = [vp]
        L.ff_synchronize.argtypes = [vp]
        for n in ("ff_statim", "ff_boundi"):
            getattr(L, n).argtypes = [vp, ci]
        L.ff_residu.argtypes = [vp, ci, ci, ci]
        L.ff_resl2.argtypes = [vp, ci, ctypes.POINTER(cd)]
        L.ff_imps.argtypes = [vp, ci, ci]
        L.ff_time_levels.argtypes = [vp, ci, ci]
        L.ff_block_metrics.argtypes = [vp, ci, vp]
        L.ff_block_metrics_levels.argtypes = [vp, ci, ci, vp]
        L.ff_wall_distance.argtypes = [vp, ci, vp, ci]
        L.ff_fin.argtypes = [vp, ci, ctypes.POINTER(cd)]
        L.ff_cycles.argtypes = [vp, ci, ci, ci, ctypes.POINTER(cd), ci]
        L.ff_time_cycles.argtypes = [vp, ci, ci, ctypes.POINTER(ctypes.c_float)]
        L.ff_time_stage.argtypes = [vp, ci, ci, ci, ctypes.POINTER(ctypes.c_float)]
        L.ff_cycle_launches.argtypes = [vp, ci]
        L.ff_lusgs_kind.argtypes = [vp, ci]
        L.ff_residual_shape.argtypes = [vp, ci]
        L.ff_sweep_tuning.argtypes = [vp, ci, ctypes.POINTER(ctypes.c_float)]
        L.ff_sweep_times.argtypes = [vp, ci, ctypes.POINTER(ctypes.c_float)]
        L.ff_host_register.argtypes = [vp, vp, ctypes.c_size_t]
        L.ff_host_unregister.argtypes = [vp, vp]
        L.ff_imps_noalloc.argtypes = [ci, ci, ci, ctypes.POINTER(FFParams), ctypes.POINTER(vp), ci, vp]
        L.ff_residi.argtypes = [vp, ci, ci, ci]
        L.ff_transf.argtypes = [vp, ci, ci]
        L.ff_forcfu.argtypes = [vp, ci]
        L.ff_addres.argtypes = [vp, ci]
        L.ff_interp.argtypes = [vp, ci, ci]
        L.ff_fortran_bind.argtypes = [vp]
        L.ff_fortran_block.argtypes = [ci, ci, ci, ci]
        L.ff_fortran_cycle.argtypes = [ci]
        L.ff_fortran_ierr.argtypes = []
        _LIB = L
    return _LIB


def _dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class GpuSolver:
    """One device context holding one or more blocks."""

    def __init__(self, device: int = 0):
        self.L = lib()
        h = ctypes.c_void_p()
        self._check(self.L.ff_create(ctypes.byref(h), device), None)
        self.ctx = h
        self.blocks = []

    def _check(self, rc, ctx="self"):
        if rc != 0:
            msg = self.L.ff_last_error(self.ctx if ctx == "self" else None)
            raise FinfloGpuError(f"libfinflo_gpu error {rc}: {msg.decode() if msg else ''}")

    def close(self):
        if getattr(self, "ctx", None):
            self.L.ff_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- blocks --------------------------------------------------------
    def add_block(self, blk: Block, prm: FFParams) -> int:
        pats = blk.patch_array()
        bid = self.L.ff_block_add(self.ctx, blk.imax, blk.jmax, blk.kmax, len(blk.patches),
                                  ctypes.cast(pats, ctypes.POINTER(FFPatch)), ctypes.byref(prm))
        if bid < 0:
            self._check(-bid)
        self.blocks.append((blk, prm))
        return bid

    def add_levels(self, levels, prms) -> int:
        """Add the multigrid levels of one block (finest first) and link
        them; returns the id of the finest level."""
        ids = [self.add_block(b, p) for b, p in zip(levels, prms)]
        for f, c in zip(ids[:-1], ids[1:]):
            self._check(self.L.ff_mg_link(self.ctx, f, c))
        self._coarse = list(getattr(self, "_coarse", [])) + ids[1:]
        return ids[0]

    def set_params(self, bid: int, prm: FFParams):
        self._check(self.L.ff_block_params(self.ctx, bid, ctypes.byref(prm)))

    def upload(self, bid: int, names=None, src=None):
        """Host -> device copies of the named slots, from the block's own
        arrays or from the dict `src`."""
        blk = self.blocks[bid][0]
        for n in names or SLOTS:
            a = src[n] if src is not None else blk.arrays[n]
            self._check(self.L.ff_upload(self.ctx, bid, SLOT[n], _dptr(a)))
        self.sync()

    def pin(self, arrays):
        """Page-lock host arrays used for every-cycle uploads/downloads;
        returns them (call unpin before they are freed)."""
        for a in arrays:
            self._check(self.L.ff_host_register(self.ctx, a.ctypes.data, a.nbytes))
        return arrays

    def unpin(self, arrays):
        for a in arrays:
            self._check(self.L.ff_host_unregister(self.ctx, a.ctypes.data))

    def download(self, bid: int, names=None, into=None) -> dict:
        blk = self.blocks[bid][0]
        out = {}
        for n in names or SLOTS:
            a = into[n] if into is not None else np.empty(blk.ntot)
            self._check(self.L.ff_download(self.ctx, bid, SLOT[n], _dptr(a)))
            out[n] = a
        self.sync()
        return out

    def device_ptr(self, bid: int, name: str) -> int:
        return self.L.ff_device_ptr(self.ctx, bid, SLOT[name])

    def sync(self):
        self._check(self.L.ff_synchronize(self.ctx))

    # ---- stages (reference routine names) -------------------------------
    def statim(self, bid=0):
        self._check(self.L.ff_statim(self.ctx, bid))

    def boundi(self, bid=0):
        self._check(self.L.ff_boundi(self.ctx, bid))

    def residu(self, bid=0, level=1, icycle=1):
        self._check(self.L.ff_residu(self.ctx, bid, level, icycle))

    def resl2(self, bid=0) -> np.ndarray:
        r = (ctypes.c_double * 5)()
        self._check(self.L.ff_resl2(self.ctx, bid, r))
        return np.array(r[:])

    def residi(self, bid, m2, icycle=1):
        """RESIDI(M, N, M2) on the block's own multigrid level."""
        self._check(self.L.ff_residi(self.ctx, bid, m2, icycle))

    def transf(self, fine, coarse):
        self._check(self.L.ff_transf(self.ctx, fine, coarse))

    def forcfu(self, bid):
        self._check(self.L.ff_forcfu(self.ctx, bid))

    def addres(self, bid):
        self._check(self.L.ff_addres(self.ctx, bid))

    def interp(self, coarse, fine):
        self._check(self.L.ff_interp(self.ctx, coarse, fine))

    def imps(self, bid=0, level=1):
        self._check(self.L.ff_imps(self.ctx, bid, level))

    def block_metrics(self, bid, X, Y, Z):
        """Metrics of the block from its nodes (arrays [nk, nj, ni]) on the device."""
        xyz = np.ascontiguousarray(np.concatenate([np.ravel(X), np.ravel(Y), np.ravel(Z)]), dtype=np.float64)
        self._check(self.L.ff_block_metrics(self.ctx, bid, xyz.ctypes.data))

    def block_metrics_levels(self, bid, nlev, X, Y, Z):
        """Metrics of the block and its nlev - 1 linked coarse levels on the device."""
        xyz = np.ascontiguousarray(np.concatenate([np.ravel(X), np.ravel(Y), np.ravel(Z)]), dtype=np.float64)
        self._check(self.L.ff_block_metrics_levels(self.ctx, bid, nlev, xyz.ctypes.data))

    def wall_distance(self, bid, pts):
        """DISTW on the device of the block and its linked coarse levels from
        the wall points pts [n, 3] (case.wall_points, PICK_XYZ)."""
        t = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
        self._check(self.L.ff_wall_distance(self.ctx, bid, t.ctypes.data if len(t) else None, len(t)))

    def time_levels(self, bid=0, mode=1):
        """TIMEL: mode 0 = STARTI (both old levels = the state), 1 = NEWTIM."""
        self._check(self.L.ff_time_levels(self.ctx, bid, mode))

    def fin(self, bid=0) -> float:
        d = ctypes.c_double()
        self._check(self.L.ff_fin(self.ctx, bid, ctypes.byref(d)))
        return d.value

    def cycles(self, n, bid=0, icycle0=1, use_graph=True) -> np.ndarray:
        hist = np.zeros((max(n, 1), 6))
        self._check(self.L.ff_cycles(self.ctx, bid, n, icycle0, _dptr(hist), int(use_graph)))
        return hist[:n]

    def halo_plan(self, items, send_ptr, recv_ptr):
        """Remote 1:1 patches: items (FFHaloItem list) and the device
        addresses of the packed send / receive buffers."""
        arr = (FFHaloItem * max(1, len(items)))(*items)
        self._check(self.L.ff_halo_plan(self.ctx, len(items), arr, ctypes.c_void_p(send_ptr or None),
                                        ctypes.c_void_p(recv_ptr or None)))

    def mb_phase(self, phase, icycle=2, use_graph=True):
        self._check(self.L.ff_mb_phase(self.ctx, phase, icycle, int(use_graph)))

    def reserve_history(self, n, reset=True):
        self._check(self.L.ff_history(self.ctx, n, None, int(reset)))

    def history(self, n, reset=False) -> np.ndarray:
        h = np.zeros((max(n, 1), 6))
        self._check(self.L.ff_history(self.ctx, n, _dptr(h), int(reset)))
        return h[:n]

    def stream_handle(self) -> int:
        return self.L.ff_stream(self.ctx) or 0

    def boundi_all(self):
        self._check(self.L.ff_boundi_all(self.ctx))

    def add_multiblock(self, block_levels, block_prms):
        """Blocks joined by 1:1 patches, each with its multigrid levels
        (finest first; a patch's IBTYPE is the source block's index in
        block_levels).  The context sees the 1:1 patches of the level-1
        blocks renumbered to its own block ids; the Block objects keep
        theirs.  Returns the ids of the level-1 blocks."""
        from . import grid
        from .case import FFPatch
        base = len(self.blocks)
        fine_ids, n = [], base
        for levels in block_levels:
            fine_ids.append(n)
            n += len(levels)
        ids = []
        for levels, prms in zip(block_levels, block_prms):
            fine = levels[0]
            orig = fine.patches
            pats = []
            for pa in orig:
                q = FFPatch.from_buffer_copy(pa)
                if q.ityp == grid.BC_CON and q.ibtype >= 0:
                    q.ibtype = fine_ids[q.ibtype]
                pats.append(q)
            fine.patches = pats
            try:
                ids.append(self.add_levels(levels, prms) if len(levels) > 1 else self.add_block(fine, prms[0]))
            finally:
                fine.patches = orig
        assert ids == fine_ids
        return ids

    def start_all(self):
        """NS3D start-up over every block: BOUNDI(1) with the 1:1
        connections, then the *OLD copies of each level-1 block."""
        self.boundi_all()
        self.sync()
        coarse = set(getattr(self, "_coarse", ()))
        for bid in range(len(self.blocks)):
            if bid not in coarse:
                self._old_copies(bid)

    def cycles_all(self, n, icycle0=1, use_graph=True) -> np.ndarray:
        """n cycles over every block (multi-block NS3D with 1:1 CONNEC)."""
        hist = np.zeros((max(n, 1), 6))
        self._check(self.L.ff_cycles_all(self.ctx, n, icycle0, _dptr(hist), int(use_graph)))
        return hist[:n]

    def time_cycles_all(self, n):
        ms = ctypes.c_float()
        nl = ctypes.c_int()
        self._check(self.L.ff_time_cycles_all(self.ctx, n, ctypes.byref(ms), ctypes.byref(nl)))
        return ms.value, nl.value

    def time_cycles(self, n, bid=0) -> float:
        ms = ctypes.c_float()
        self._check(self.L.ff_time_cycles(self.ctx, bid, n, ctypes.byref(ms)))
        return ms.value

    def residual_shape(self, bid=0) -> str:
        return ("32x4x4", "16x8x4", "8x8x8", "32x4x4 staged", "16x8x4 staged",
                "8x8x8 staged")[self.L.ff_residual_shape(self.ctx, bid)]

    def lusgs_kind(self, bid=0) -> int:
        return self.L.ff_lusgs_kind(self.ctx, bid)

    def sweep_tuning(self, bid=0):
        ms = (ctypes.c_float * 3)()
        self._check(self.L.ff_sweep_times(self.ctx, bid, ms))
        return {"pipe_ms": ms[0], "lines_ms": ms[1], "hyperplane_ms": ms[2]}

    def cycle_launches(self, bid=0) -> int:
        return self.L.ff_cycle_launches(self.ctx, bid)

    def time_stage(self, stage, reps=10, bid=0) -> float:
        ms = ctypes.c_float()
        self._check(self.L.ff_time_stage(self.ctx, bid, stage, reps, ctypes.byref(ms)))
        return ms.value

    def start(self, bid=0):
        """NS3D start-up (ns3c.f:378-379): BOUNDI, then the *OLD copies."""
        self.boundi(bid)
        self.sync()
        self._old_copies(bid)

    def _old_copies(self, bid):
        blk = self.blocks[bid][0]
        st = self.download(bid, ["TEMP", "U", "V", "W", "PDIFF"])
        pairs = [("TOLD", "TEMP"), ("UOLD", "U"), ("VOLD", "V"), ("WOLD", "W"), ("POLD", "PDIFF")]
        if self.blocks[bid][1].iturb >= 3:
            pairs += [("RKOLD", "RK"), ("EPSOLD", "REPS")]
            st.update(self.download(bid, ["RK", "REPS"]))
        for a, b2 in pairs:   # device copies; the host block keeps a copy when it still has arrays
            self._check(self.L.ff_upload(self.ctx, bid, SLOT[a], _dptr(st[b2])))
            if a in blk.arrays:
                blk.arrays[a][:] = st[b2]
        self.sync()
