"""The allocation-free implicit stage (ff_imps_noalloc) against ff_imps.

ff_imps_noalloc serves callers that cannot allocate device memory while they
run (a host whose device memory is all owned by its own pool, or one under a
fixed memory cap): it takes the caller's device arrays and keeps its LU-SGS
scratch in a fixed file-scope device array.  This test feeds it the same
residual as the context-based ff_imps and requires the same increments and
local time steps (the two run the same kernels, so the tolerance of the other
LU-SGS parity tests, 1e-12 relative, is ample), on two calls in a row.  The
file name sorts last so a run that stops at the first failure has already run
every other test.
"""
import ctypes

import numpy as np
import pytest

from finflo_b200 import case
from finflo_b200.case import FFParams, SLOT, SLOTS
from finflo_b200.gpu import GpuSolver
from tests.util import interior

pytestmark = pytest.mark.gpu

RES = ["DRO", "DM", "DN", "DW", "DE"]
FF_ERR_ARG = 2
FF_ERR_SIZE = 4
FF_NOALLOC_MAX_NTOT = 98304


def _slots(g, bid):
    arr = (ctypes.c_void_p * len(SLOTS))()
    for i, n in enumerate(SLOTS):
        arr[i] = g.device_ptr(bid, n)
    return arr


@pytest.mark.parametrize("ddadi", [0, 1])
def test_imps_noalloc_matches_imps_twice(gpu_lib, ddadi):
    """LU-SGS, and the DDADI line sweeps (LUSGS=0), which need no scratch."""
    blk, prm, fs = case.bump_case(33, 17, 17)          # 32x16x16 cells, NTOT = 29,160
    prm.ddadi = ddadi
    g = GpuSolver(0)
    bid = g.add_block(blk, prm)
    g.upload(bid)
    g.start(bid)
    g.statim(bid)
    g.residu(bid, 1, 1)
    g.sync()
    res0 = g.download(bid, RES)
    res0 = {n: a.copy() for n, a in res0.items()}
    slots = _slots(g, bid)
    L = g.L
    stream = L.ff_stream(g.ctx)
    for call in range(2):
        # reference: the context-based stage
        for n in RES:
            blk.arrays[n][:] = res0[n]
        g.upload(bid, RES)
        g.imps(bid, 1)
        g.sync()
        ref = {n: a.copy() for n, a in g.download(bid, RES + ["DTL"]).items()}
        # the allocation-free stage on the same inputs
        g.upload(bid, RES)
        rc = L.ff_imps_noalloc(blk.imax, blk.jmax, blk.kmax, ctypes.byref(prm),
                               ctypes.cast(slots, ctypes.POINTER(ctypes.c_void_p)), 1, stream)
        assert rc == 0, rc
        g.sync()
        got = g.download(bid, RES + ["DTL"])
        for n in RES + ["DTL"]:
            a, b = interior(blk, got[n]), interior(blk, ref[n])
            err = np.abs(a - b).max() / (np.abs(b).max() + 1e-300)
            assert err <= 1e-12, (call, n, err)
    # the status query (level 0): no sweep of these calls timed out
    assert L.ff_imps_noalloc(0, 0, 0, None, None, 0, stream) == 0
    g.close()


def test_imps_noalloc_refuses_fp32_lusgs(gpu_lib):
    """Its LU-SGS sweeps are FP64 only: an FP32 request is refused, not
    silently run in FP64."""
    L = gpu_lib
    blk, prm, fs = case.bump_case(17, 9, 9)
    prm.lusgs_fp32 = 1
    slots = (ctypes.c_void_p * len(SLOTS))(*([1] * len(SLOTS)))
    rc = L.ff_imps_noalloc(blk.imax, blk.jmax, blk.kmax, ctypes.byref(prm),
                           ctypes.cast(slots, ctypes.POINTER(ctypes.c_void_p)), 1, None)
    assert rc == FF_ERR_ARG


def test_imps_noalloc_rejects_oversized_block(gpu_lib):
    """A block above FF_NOALLOC_MAX_NTOT is refused before any GPU work."""
    L = gpu_lib
    prm = FFParams()
    slots = (ctypes.c_void_p * len(SLOTS))()
    # 64x64x32 cells: (68*68*36) = 166,464 > FF_NOALLOC_MAX_NTOT
    rc = L.ff_imps_noalloc(64, 64, 32, ctypes.byref(prm), ctypes.cast(slots, ctypes.POINTER(ctypes.c_void_p)),
                           1, None)
    assert rc == FF_ERR_SIZE
    assert (64 + 4) * (64 + 4) * (32 + 4) > FF_NOALLOC_MAX_NTOT
