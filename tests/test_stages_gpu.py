"""The multigrid stage entry points (ff_residi, ff_transf, ff_forcfu,
ff_addres, ff_interp, coarse-level ff_imps / ff_fin) and the Fortran
call-site wrappers (statim_, residi_, impsdi_, fin_, boundi_), each against
the oracle on the same inputs.

Every stage gets identical inputs on both sides (the GPU's arrays are copied
into the oracle's block first), so each comparison isolates one stage:
TRANSF multi.f:156, FORCFU multi.f:1609, ADDRES multi.f:1686, INTERP
multi.f:1763 (+ INTERT multi.f:2051 and the limits of ns3c.f:2059-2125).
"""
import ctypes

import numpy as np
import pytest

from finflo_b200 import case
from finflo_b200.case import SLOTS
from finflo_b200.gpu import GpuSolver
from oracle.oracle import Oracle
from tests.util import interior

pytestmark = pytest.mark.gpu

SST = dict(turbulence="sst", reynolds=1e6, mach=0.6, h1=1e-4)
RES5 = ["DRO", "DM", "DN", "DW", "DE"]
RES7 = RES5 + ["DRK", "DEPS"]
P2H5 = ["ROP2H", "RMP2H", "RNP2H", "RWP2H", "EP2H"]
P2H7 = P2H5 + ["RKP2H", "EPP2H"]


def _pair(sst):
    kw = SST if sst else {}
    lg, pg, fs = case.bump_case_mg(17, 9, 9, nlev=2, **kw)
    lc, pc, _ = case.bump_case_mg(17, 9, 9, nlev=2, **kw)
    g = GpuSolver(0)
    f = g.add_levels(lg, pg)
    c = f + 1
    g.upload(f)
    g.upload(c)
    g.start(f)
    of, oc = Oracle(lc[0], pc[0]), Oracle(lc[1], pc[1])
    return g, f, c, lg, lc, of, oc


def _to_oracle(g, bid, blk_c, names=None):
    """Copy the device arrays of block bid into the oracle's block."""
    d = g.download(bid, names or SLOTS)
    for n, a in d.items():
        blk_c.arrays[n][:] = a


def _cmp(g, bid, blk_c, names, rtol, ring=False):
    """ring: compare the interior and the first ghost layer only.  TRANSF
    computes those cells; the second ghost layer copies the first along each
    face normal, and its edge and corner cells (second layer in two
    directions), which coarse levels never read, are filled in a different
    order on the two sides."""
    d = g.download(bid, names)
    for n in names:
        ref, got = blk_c.arrays[n], d[n]
        if ring:
            shp = (blk_c.kmax + 4, blk_c.jmax + 4, blk_c.imax + 4)
            ref, got = ref.reshape(shp)[1:-1, 1:-1, 1:-1], got.reshape(shp)[1:-1, 1:-1, 1:-1]
        err = np.abs(got - ref).max() / (np.abs(ref).max() + 1e-300)
        assert err <= rtol, (n, err)


@pytest.mark.parametrize("sst", [False, True])
def test_multigrid_stages_match_oracle(gpu_lib, sst):
    g, f, c, lg, lc, of, oc = _pair(sst)
    L = of.L
    # RESIDI(1, N, 2) of the fine level, then TRANSF (TRANKE)
    g.statim(f)
    g.residi(f, 2, 1)
    g.sync()
    _to_oracle(g, f, lc[0])
    _to_oracle(g, c, lc[1])
    g.transf(f, c)
    L.orc_transf(ctypes.byref(of.ob), ctypes.byref(oc.ob))
    if sst:
        L.orc_tranke(ctypes.byref(of.ob), ctypes.byref(oc.ob))
    vs = ["TEMP", "U", "V", "W", "PDIFF", "EPS2", "VIST", "TOLD", "UOLD", "VOLD", "WOLD", "POLD"]
    if sst:
        vs += ["RK", "REPS", "RKOLD", "EPSOLD"]
    _cmp(g, c, lc[1], vs, 1e-14, ring=True)
    _cmp(g, c, lc[1], P2H7 if sst else P2H5, 1e-14)
    # the coarse residual RESIDI(2, N, 2), then FORCFU and ADDRES
    g.statim(c)
    g.residu(c, 2, 1)
    g.sync()
    _to_oracle(g, c, lc[1])
    g.forcfu(c)
    (L.orc_forcfu_ke if sst else L.orc_forcfu)(ctypes.byref(oc.ob))
    _cmp(g, c, lc[1], P2H7 if sst else P2H5, 1e-14)
    g.addres(c)
    (L.orc_addres_ke if sst else L.orc_addres)(ctypes.byref(oc.ob))
    _cmp(g, c, lc[1], RES7 if sst else RES5, 1e-14)
    # the coarse implicit stage and FIN, then INTERP (INTERT) + limits
    g.imps(c, 2)
    g.fin(c)
    g.sync()
    _to_oracle(g, c, lc[1])
    _to_oracle(g, f, lc[0])
    g.interp(c, f)
    L.orc_interp_limits(ctypes.byref(oc.ob), ctypes.byref(of.ob), ctypes.byref(of.prm))
    fs = ["TEMP", "U", "V", "W", "PDIFF", "P"] + (["RK", "REPS"] if sst else [])
    _cmp(g, f, lc[0], fs, 1e-14)
    g.close()


def test_coarse_level_residual_and_implicit_stage_match_oracle(gpu_lib):
    """RESIDI(2, N, 2) (first-order Roe, FLUXDO) and IMPSDI on level 2."""
    g, f, c, lg, lc, of, oc = _pair(False)
    g.statim(f)
    g.residi(f, 2, 1)
    g.transf(f, c)
    g.statim(c)
    g.sync()
    _to_oracle(g, c, lc[1])
    g.residu(c, 2, 1)
    oc.residu(2, 1)
    _cmp(g, c, lc[1], RES5, 1e-11)
    g.sync()
    _to_oracle(g, c, lc[1], RES5)
    g.imps(c, 2)
    oc.imps(2)
    _cmp(g, c, lc[1], RES5 + ["DTL"], 1e-11)
    g.close()


def test_fortran_wrappers_run_a_cycle_like_the_oracle(gpu_lib):
    """A Fortran host's single-grid cycle through the gfortran-named
    wrappers: STATIM(1,N,0,.TRUE.), RESIDI(1,N,1,IPR), IMPSDI(1,N,1,AMG),
    FIN(...,NGL,ICYCLE), BOUNDI(1) against the oracle's cycle."""
    blk_g, prm, fs = case.bump_case(17, 9, 9)
    blk_c, _, _ = case.bump_case(17, 9, 9)
    o = Oracle(blk_c, prm)
    o.start()
    g = GpuSolver(0)
    bid = g.add_block(blk_g, prm)
    g.upload(bid)
    g.start(bid)
    L = g.L
    i = ctypes.c_int
    assert L.ff_fortran_bind(g.ctx) == 0
    assert L.ff_fortran_block(1, 1, 7, bid) == 0           # level 1, block 1, global block 7
    one, yes, ngl = i(1), i(1), i(7)
    amg = ctypes.c_double(0.0)
    imax, jmax, kmax = i(blk_g.imax), i(blk_g.jmax), i(blk_g.kmax)
    null = ctypes.c_void_p()
    for cyc in range(1, 4):
        L.ff_fortran_cycle(cyc)
        L.statim_(ctypes.byref(one), ctypes.byref(one), ctypes.byref(i(0)), ctypes.byref(yes))
        L.residi_(ctypes.byref(one), ctypes.byref(one), ctypes.byref(one), ctypes.byref(one))
        L.impsdi_(ctypes.byref(one), ctypes.byref(one), ctypes.byref(one), ctypes.byref(amg))
        args = [null] * 21 + [ctypes.byref(ctypes.c_double(0.0))] * 2 + [null] * 7 \
            + [ctypes.byref(imax), ctypes.byref(jmax), ctypes.byref(kmax)] + [ctypes.byref(i(0))] * 5 \
            + [ctypes.byref(ctypes.c_double(0.0)), null, ctypes.byref(i(0)), null, null,
               ctypes.byref(ngl), ctypes.byref(i(cyc))]
        assert len(args) == 45
        L.fin_(*args)
        L.boundi_(ctypes.byref(one))
        assert L.ff_fortran_ierr() == 0
        o.cycle(cyc)
    g.sync()
    d = g.download(bid, ["TEMP", "U", "V", "W", "PDIFF"])
    for n in d:
        a, b = interior(blk_g, d[n]), interior(blk_c, blk_c.arrays[n])
        rel = np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-300)
        assert rel <= 1e-10, (n, rel)
    # an unknown block is reported through ff_fortran_ierr, not by aborting
    L.residi_(ctypes.byref(i(2)), ctypes.byref(one), ctypes.byref(i(2)), ctypes.byref(one))
    assert L.ff_fortran_ierr() == 2
    assert L.ff_fortran_ierr() == 0
    g.close()
