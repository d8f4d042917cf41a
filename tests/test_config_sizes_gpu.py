"""Parity at the workloads' own grids and geometry (not only small blocks).

* the laminar bump channel at 64x32x32 cells (65x33x33 nodes, first cell
  1e-3, Re 1e4, M 0.5): one residual, one implicit stage, five cycles;
* the k-omega SST bump channel at 128x64x64 cells (129x65x65 nodes, first
  cell 2e-6, Re 1e6, M 0.6), where the high-aspect wall cells and the BOTSKE
  wall faces dominate: one residual, one implicit stage, two 3-level
  V-cycles, and one V-cycle with the FP32 implicit stage on every level,
  whose fields are reported against the FP64 oracle's;
* a residual with the entropy fix (ENTROPY_FIX, base3c.f:5040).

Tolerances as in the small-block tests: residual 1e-12 of max(|R|, S) per
cell, implicit stage 1e-11, cycle histories 1e-8 (1e-7 for the V-cycles),
fields after the cycles 1e-10 (1e-9).
"""
import numpy as np
import pytest

from finflo_b200 import case
from finflo_b200.gpu import GpuSolver
from oracle.oracle import Oracle, OracleMG
from tests.util import flux_scale, flux_scale_sst, interior, make_pair

pytestmark = pytest.mark.gpu

RES5 = ("DRO", "DM", "DN", "DW", "DE")
RES7 = RES5 + ("DRK", "DEPS")
C2 = dict(turbulence="sst", reynolds=1e6, mach=0.6, h1=2e-6, noise=1e-3, seed=1)


def _hist_close(got, ref, rtol):
    """Residual-norm histories (sums of squares of DRO, DM, DN, DW, DE): the
    spanwise momentum residual is zero up to rounding in these
    spanwise-uniform cases, so the momentum components share one scale."""
    mom = ref[:, 1:4].max()
    for c in range(5):
        atol = rtol * mom if c in (1, 2, 3) else 0.0
        np.testing.assert_allclose(got[:, c], ref[:, c], rtol=rtol, atol=atol)


def _residual_check(bg, bc, got, S, names):
    for n in names:
        ref = interior(bc, bc.arrays[n]); g = interior(bg, got[n])
        den = np.maximum(np.abs(ref), S[n]) + 1e-300
        err = (np.abs(g - ref) / den).max()
        assert err <= 1e-12, (n, err)


def test_laminar_workload_grid(gpu_lib):
    bg, bc, prm, fs = make_pair(65, 33, 33)
    o = Oracle(bc, prm)
    o.start()
    g = GpuSolver(0)
    bid = g.add_block(bg, prm)
    g.upload(bid)
    g.start(bid)
    o.statim(); o.adjuin(); o.residu(1, 1)
    g.residu(bid, 1, 1)
    g.sync()
    got = g.download(bid, list(RES5))
    _residual_check(bg, bc, got, flux_scale(o, bc), RES5)
    for n in RES5:
        bc.arrays[n][:] = got[n]
    o.imps(1)
    g.imps(bid, 1)
    g.sync()
    d = g.download(bid, list(RES5) + ["DTL"])
    for n in list(RES5) + ["DTL"]:
        ref = interior(bc, bc.arrays[n]); x = interior(bg, d[n])
        err = np.abs(x - ref).max() / (np.abs(ref).max() + 1e-300)
        assert err <= 1e-11, (n, err)
    g.close()
    # five whole cycles from the start on both sides
    bg, bc, prm, fs = make_pair(65, 33, 33)
    o = Oracle(bc, prm)
    o.start()
    g = GpuSolver(0)
    bid = g.add_block(bg, prm)
    g.upload(bid)
    g.start(bid)
    hist = g.cycles(5, bid, icycle0=1)
    ref = np.array([o.cycle(i + 1)[0] for i in range(5)])
    _hist_close(hist[:, :5], ref, 1e-8)
    d = g.download(bid, ["TEMP", "U", "V", "W", "PDIFF"])
    for n in d:
        a, b = interior(bg, d[n]), interior(bc, bc.arrays[n])
        scale = np.linalg.norm(interior(bc, bc.arrays["U"])) if n == "W" else np.linalg.norm(b)
        rel = np.linalg.norm(a - b) / (scale + 1e-300)
        assert rel <= 1e-10, (n, rel)
    g.close()


def test_sst_workload_grid_residual_and_implicit_stage(gpu_lib):
    bg, bc, prm, fs = make_pair(129, 65, 65, **C2)
    o = Oracle(bc, prm)
    o.start()
    g = GpuSolver(0)
    bid = g.add_block(bg, prm)
    g.upload(bid)
    g.start(bid)
    o.statim(); o.turbeq(); o.residu_sst(1)
    g.statim(bid); g.residu(bid, 1, 1)
    g.sync()
    got = g.download(bid, list(RES7))
    _residual_check(bg, bc, got, flux_scale_sst(o, bc), RES7)
    for n in RES7:
        bc.arrays[n][:] = got[n]
    o.imps_sst()
    g.imps(bid, 1)
    g.sync()
    d = g.download(bid, list(RES7) + ["DTL"])
    for n in list(RES7) + ["DTL"]:
        ref = interior(bc, bc.arrays[n]); x = interior(bg, d[n])
        err = np.abs(x - ref).max() / (np.abs(ref).max() + 1e-300)
        assert err <= 1e-11, (n, err)
    g.close()


def _mg_pair(fp32=0):
    lg, pg, fs = case.bump_case_mg(129, 65, 65, nlev=3, **C2)
    lc, pc, _ = case.bump_case_mg(129, 65, 65, nlev=3, **C2)
    om = OracleMG(lc, pc)
    om.start()
    for q in pg:
        q.lusgs_fp32 = fp32
    g = GpuSolver(0)
    bid = g.add_levels(lg, pg)
    for b in range(len(lg)):
        g.upload(bid + b)
    g.start(bid)
    return g, bid, lg, lc, om


def test_sst_workload_grid_vcycles(gpu_lib):
    g, bid, lg, lc, om = _mg_pair()
    n = 2
    hist = g.cycles(n, bid, icycle0=1)
    ref = np.array([om.cycle(i + 1)[0] for i in range(n)])
    _hist_close(hist[:, :5], ref, 1e-7)
    d = g.download(bid, ["TEMP", "U", "V", "PDIFF", "RK", "REPS"])
    for nme in d:
        a, b = interior(lg[0], d[nme]), interior(lc[0], lc[0].arrays[nme])
        rel = np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-300)
        assert rel <= 1e-9, (nme, rel)
    g.close()


def test_sst_workload_grid_fp32_vcycle_error(gpu_lib):
    """One V-cycle with the FP32 implicit stage on every level against the
    FP64 oracle: the fields differ by the FP32 rounding of one increment."""
    g, bid, lg, lc, om = _mg_pair(fp32=1)
    g.cycles(1, bid, icycle0=1)
    om.cycle(1)
    d = g.download(bid, ["TEMP", "U", "V", "PDIFF", "RK", "REPS"])
    errs = {}
    for nme in d:
        a, b = interior(lg[0], d[nme]), interior(lc[0], lc[0].arrays[nme])
        errs[nme] = np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-300)
    print("FP32 implicit stage, one V-cycle, relative L2 against the FP64 oracle:", errs)
    # the state itself moves by ~1e-3 of its size per cycle; its FP32
    # increment carries ~1e-7 of that
    assert max(errs.values()) <= 1e-6, errs
    g.close()


def test_entropy_fix_residual(gpu_lib):
    """ENTROPY_FIX (base3c.f:5040) residual after a few cycles, 1e-12."""
    bg, bc, prm, fs = make_pair(33, 17, 9)
    prm.entropy_fix = 1
    o = Oracle(bc, prm)
    o.start()
    g = GpuSolver(0)
    bid = g.add_block(bg, prm)
    g.upload(bid)
    g.start(bid)
    g.cycles(5, bid, icycle0=1, use_graph=False)
    for i in range(5):
        o.cycle(i + 1)
    d = g.download(bid)
    for n, a in d.items():
        bc.arrays[n][:] = a
    o.statim(); o.adjuin(); o.residu(1, 6)
    g.statim(bid); g.residu(bid, 1, 6)
    g.sync()
    got = g.download(bid, list(RES5))
    _residual_check(bg, bc, got, flux_scale(o, bc), RES5)
    # the fix changes the residual (it is active somewhere)
    prm0 = type(prm).from_buffer_copy(prm)
    prm0.entropy_fix = 0
    o0 = Oracle(bc, prm0)
    o0.statim(); o0.adjuin(); o0.residu(1, 6)
    diff = max(np.abs(interior(bc, bc.arrays[n]) - interior(bg, got[n])).max() for n in RES5)
    assert diff > 0.0
    g.close()
