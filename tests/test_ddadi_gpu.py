"""DDADI implicit stage (LUSGS=0) on the sm_100a path against the CPU oracle:
the k, i and j line sweeps (PRED + DIAG, CORR) for the laminar and the
k-omega SST equations, FP64 and FP32, alone and inside full cycles."""
import numpy as np
import pytest

from finflo_b200.gpu import GpuSolver
from oracle.oracle import Oracle
from tests.util import hist_close, interior, make_pair

pytestmark = pytest.mark.gpu

RES5 = ("DRO", "DM", "DN", "DW", "DE")
RES7 = RES5 + ("DRK", "DEPS")
SST = dict(turbulence="sst", reynolds=1e6, mach=0.6, h1=1e-4)


def _setup(dims, fp32=False, **kw):
    bg, bc, prm, fs = make_pair(*dims, **kw)
    prm.ddadi = 1
    prm.lusgs_fp32 = int(fp32)
    o = Oracle(bc, prm)
    o.start()
    g = GpuSolver(0)
    bid = g.add_block(bg, prm)
    g.upload(bid)
    g.start(bid)
    return g, bid, bg, o, bc, prm


def _imps_case(dims, sst, fp32=False):
    """The same residual on both sides, then one implicit stage; returns the
    worst relative error over the increments and DTL."""
    kw = SST if sst else {}
    res = RES7 if sst else RES5
    g, bid, bg, o, bc, prm = _setup(dims, fp32=fp32, **kw)
    if sst:
        o.statim(); o.turbeq(); o.residu_sst(1)
    else:
        o.statim(); o.adjuin(); o.residu(1, 1)
    g.residu(bid, 1, 1)
    g.sync()
    r = g.download(bid, list(res))
    for n in res:
        bc.arrays[n][:] = r[n]
    if sst:
        o.imps_sst()
    else:
        o.imps(1)
    g.imps(bid, 1)
    g.sync()
    d = g.download(bid, list(res) + ["DTL"])
    errs = {}
    for n in list(res) + ["DTL"]:
        ref = interior(bc, bc.arrays[n]); got = interior(bg, d[n])
        assert np.isfinite(got).all(), n
        errs[n] = np.abs(got - ref).max() / (np.abs(ref).max() + 1e-300)
    g.close()
    return errs


@pytest.mark.parametrize("dims", [(17, 9, 9), (33, 17, 9), (65, 33, 33), (17, 9, 3)])
def test_ddadi_imps(gpu_lib, dims):
    """Laminar PRED/DIAG/CORR along k, i, j lines (65 x 33 x 33 nodes: many
    CTAs and a partial last CTA of lines; 17 x 9 x 3: two-cell k lines)."""
    for n, e in _imps_case(dims, sst=False).items():
        assert e <= 1e-11, (n, e)


@pytest.mark.parametrize("dims", [(17, 9, 9), (33, 17, 9)])
def test_ddadi_imps_sst(gpu_lib, dims):
    """PREDKE/DIAGKE/CORRKE (SYIKE/SYM1KE) after LOCDTK/IMSOKO/COPRKE."""
    for n, e in _imps_case(dims, sst=True).items():
        assert e <= 1e-11, (n, e)


@pytest.mark.parametrize("sst", [False, True])
def test_ddadi_fp32_imps(gpu_lib, sst):
    """The same sweeps with FP32 arithmetic: increments within FP32 rounding
    of the FP64 oracle."""
    errs = _imps_case((33, 17, 9), sst=sst, fp32=True)
    for n, e in errs.items():
        assert e <= (1e-11 if n == "DTL" else 2e-4), (n, e)


@pytest.mark.parametrize("use_graph", [False, True])
def test_ddadi_cycles_match_oracle(gpu_lib, use_graph):
    """30 full laminar cycles with the DDADI stage: residual history and fields."""
    g, bid, bg, o, bc, prm = _setup((17, 9, 9))
    n = 30
    hist = g.cycles(n, bid, icycle0=1, use_graph=use_graph)
    ref = np.array([o.cycle(i + 1)[0] for i in range(n)])
    hist_close(hist[:, :5], ref, 1e-8)
    d = g.download(bid, ["TEMP", "U", "V", "W", "PDIFF"])
    for nme in d:
        a = interior(bg, d[nme]); b = interior(bc, bc.arrays[nme])
        rel = np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-300)
        assert rel <= 1e-10, (nme, rel)
    g.close()


def test_ddadi_sst_cycles_match_oracle(gpu_lib):
    """25 SST cycles with the DDADI stage, k and omega included."""
    g, bid, bg, o, bc, prm = _setup((17, 9, 9), **SST)
    n = 25
    hist = g.cycles(n, bid, icycle0=1, use_graph=True)
    ref = np.array([o.cycle(i + 1)[0] for i in range(n)])
    hist_close(hist[:, :5], ref, 1e-8)
    d = g.download(bid, ["TEMP", "U", "V", "W", "RK", "REPS"])
    for nme in d:
        a = interior(bg, d[nme]); b = interior(bc, bc.arrays[nme])
        rel = np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-300)
        assert rel <= 1e-10, (nme, rel)
    g.close()


@pytest.mark.parametrize("turb", [None, "sst"])
def test_ddadi_multigrid_matches_oracle(gpu_lib, turb):
    """Two-level FAS V-cycles with DDADI on both levels."""
    from finflo_b200 import case
    from oracle.oracle import OracleMG
    kw = dict(SST) if turb else {}
    lv_g, prms, fs = case.bump_case_mg(33, 17, 17, nlev=2, **kw)
    lv_c, _, _ = case.bump_case_mg(33, 17, 17, nlev=2, **kw)
    for q in prms:
        q.ddadi = 1
    om = OracleMG(lv_c, prms)
    om.start()
    g = GpuSolver(0)
    bid = g.add_levels(lv_g, prms)
    for b in range(len(lv_g)):
        g.upload(bid + b)
    g.start(bid)
    n = 10
    hist = g.cycles(n, bid, icycle0=1, use_graph=True)
    ref = np.array([om.cycle(i + 1)[0] for i in range(n)])
    hist_close(hist[:, :5], ref, 1e-7)
    d = g.download(bid, ["TEMP", "U", "V", "PDIFF"])
    for nme in d:
        a = interior(lv_g[0], d[nme]); b = interior(lv_c[0], lv_c[0].arrays[nme])
        rel = np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-300)
        assert rel <= 1e-9, (nme, rel)
    g.close()
