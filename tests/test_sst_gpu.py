"""k-omega SST (ITURB=6) on the sm_100a path against the CPU oracle."""
import numpy as np
import pytest

from finflo_b200.gpu import GpuSolver
from oracle.oracle import Oracle
from tests.util import hist_close, flux_scale_sst, interior, make_pair

pytestmark = pytest.mark.gpu

RES7 = ("DRO", "DM", "DN", "DW", "DE", "DRK", "DEPS")
SST = dict(turbulence="sst", reynolds=1e6, mach=0.6, h1=1e-4)


def _setup(dims=(17, 9, 9), **kw):
    args = dict(SST, **kw)
    bg, bc, prm, fs = make_pair(*dims, **args)
    o = Oracle(bc, prm)
    o.start()
    g = GpuSolver(0)
    bid = g.add_block(bg, prm)
    g.upload(bid)
    g.start(bid)
    return g, bid, bg, o, bc, prm


def _run_oracle_cycles(o, n):
    return np.array([o.cycle(i + 1)[0] for i in range(n)])


@pytest.mark.parametrize("dims", [(17, 9, 9), (33, 17, 9)])
def test_sst_residual(gpu_lib, dims):
    """TURBEQ + RESIKE: the seven residuals per cell within 1e-12 of
    max(|R|, S), after a few cycles so that k, omega and mu_t vary."""
    g, bid, bg, o, bc, prm = _setup(dims)
    _run_oracle_cycles(o, 5)
    g.cycles(5, bid, icycle0=1, use_graph=False)
    # same state on both sides, then one residual evaluation
    d = g.download(bid)
    for n, a in d.items():
        bc.arrays[n][:] = a
    o.statim(); o.turbeq(); o.residu_sst(6)
    g.statim(bid); g.residu(bid, 1, 6)
    g.sync()
    got_all = g.download(bid, list(RES7) + ["EPS2", "VIST", "FUN1", "PTUR"])
    S = flux_scale_sst(o, bc)
    for n in RES7:
        ref = interior(bc, bc.arrays[n]); got = interior(bg, got_all[n])
        den = np.maximum(np.abs(ref), S[n]) + 1e-300
        err = (np.abs(got - ref) / den).max()
        assert err <= 1e-12, (n, err)
    for n in ("EPS2", "VIST", "FUN1", "PTUR"):
        ref = interior(bc, bc.arrays[n]); got = interior(bg, got_all[n])
        err = np.abs(got - ref).max() / (np.abs(ref).max() + 1e-300)
        assert err <= 1e-11, (n, err)
    g.close()


@pytest.mark.parametrize("dims", [(17, 9, 9), (25, 13, 7)])
def test_sst_imps(gpu_lib, dims):
    """Seven-equation LU-SGS (PRKEGS without PREDGS's row quirk, DIKEGS,
    COKEGS) after LOCDTK/IMSOKO/COPRKE, both sweep kernels."""
    g, bid, bg, o, bc, prm = _setup(dims)
    o.statim(); o.turbeq(); o.residu_sst(1)
    g.residu(bid, 1, 1)
    g.sync()
    r = g.download(bid, list(RES7))
    for n in RES7:
        bc.arrays[n][:] = r[n]
    o.imps_sst()
    g.imps(bid, 1)
    g.sync()
    d = g.download(bid, list(RES7) + ["DTL"])
    for n in list(RES7) + ["DTL"]:
        ref = interior(bc, bc.arrays[n]); got = interior(bg, d[n])
        err = np.abs(got - ref).max() / (np.abs(ref).max() + 1e-300)
        assert err <= 1e-11, (n, err)
    g.close()


@pytest.mark.parametrize("use_graph", [False, True])
def test_sst_cycles_match_oracle(gpu_lib, use_graph):
    """40 full SST cycles: residual history and fields incl. k and omega."""
    g, bid, bg, o, bc, prm = _setup((17, 9, 9))
    n = 40
    hist = g.cycles(n, bid, icycle0=1, use_graph=use_graph)
    ref = _run_oracle_cycles(o, n)
    hist_close(hist[:, :5], ref, 1e-8)
    d = g.download(bid, ["TEMP", "U", "V", "W", "RK", "REPS", "VIST"])
    for nme in d:
        a = interior(bg, d[nme]); b = interior(bc, bc.arrays[nme])
        rel = np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-300)
        assert rel <= 1e-10, (nme, rel)
    g.close()


def test_sst_line_and_hyperplane_sweeps_agree(gpu_lib, monkeypatch):
    g1, b1, bg1, o, bc, prm = _setup((33, 33, 17))
    assert g1.lusgs_kind(b1) % 100 == 1
    monkeypatch.setenv("FINFLO_LUSGS", "hyperplane")
    g2 = GpuSolver(0)
    bg2 = make_pair(33, 33, 17, **SST)[0]
    b2 = g2.add_block(bg2, prm)
    assert g2.lusgs_kind(b2) % 100 == 2
    g2.upload(b2)
    g2.start(b2)
    for g, b in ((g1, b1), (g2, b2)):
        g.residu(b, 1, 1)
        g.imps(b, 1)
    d1 = g1.download(b1, list(RES7))
    d2 = g2.download(b2, list(RES7))
    for n in RES7:
        a, c = interior(bg1, d1[n]), interior(bg2, d2[n])
        err = np.abs(a - c).max() / (np.abs(c).max() + 1e-300)
        assert err <= 1e-12, (n, err)
    g1.close(); g2.close()


@pytest.mark.parametrize("fp32", [False, True])
def test_sst_pipe_and_hyperplane_sweeps_agree(gpu_lib, monkeypatch, fp32):
    """Seven-equation pipelined tile-wavefront sweeps against the cooperative
    hyperplane kernel, FP64 and FP32."""
    monkeypatch.setenv("FINFLO_LUSGS", "pipe")
    bg1, bc, prm, fs = make_pair(33, 33, 17, **SST)
    prm.lusgs_fp32 = int(fp32)
    g1 = GpuSolver(0)
    b1 = g1.add_block(bg1, prm)
    assert g1.lusgs_kind(b1) % 100 == 3
    g1.upload(b1)
    g1.start(b1)
    monkeypatch.setenv("FINFLO_LUSGS", "hyperplane")
    g2 = GpuSolver(0)
    bg2 = make_pair(33, 33, 17, **SST)[0]
    b2 = g2.add_block(bg2, prm)
    assert g2.lusgs_kind(b2) % 100 == 2
    g2.upload(b2)
    g2.start(b2)
    for g, b in ((g1, b1), (g2, b2)):
        g.residu(b, 1, 1)
        g.imps(b, 1)
    d1 = g1.download(b1, list(RES7))
    d2 = g2.download(b2, list(RES7))
    for n in RES7:
        a, c = interior(bg1, d1[n]), interior(bg2, d2[n])
        err = np.abs(a - c).max() / (np.abs(c).max() + 1e-300)
        assert err <= (1e-5 if fp32 else 1e-12), (n, err)
    g1.close(); g2.close()


def test_sst_fp32_lusgs_tracks_fp64(gpu_lib):
    """FP32 seven-equation implicit operator: same fixed point, bounded
    difference from the FP64 run after the same cycles."""
    g, bid, bg, o, bc, prm = _setup((17, 9, 9))
    prm32 = type(prm).from_buffer_copy(prm)
    prm32.lusgs_fp32 = 1
    g2 = GpuSolver(0)
    bg2 = make_pair(17, 9, 9, **SST)[0]
    b2 = g2.add_block(bg2, prm32)
    g2.upload(b2)
    g2.start(b2)
    h64 = g.cycles(100, bid)
    h32 = g2.cycles(100, b2)
    assert np.isfinite(h32).all()
    d64 = g.download(bid, ["TEMP", "U", "RK"])
    d32 = g2.download(b2, ["TEMP", "U", "RK"])
    for n in d64:
        a, b = interior(bg, d64[n]), interior(bg2, d32[n])
        assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-3, n
    g.close(); g2.close()


@pytest.mark.parametrize("nlev,dims", [(2, (17, 9, 9)), (3, (33, 17, 17))])
def test_sst_multigrid_cycles_match_oracle(gpu_lib, nlev, dims):
    """SST FAS V-cycles (TRANKE, k-omega forcing, coarse RESIKE with FLUDKE
    and first-order Roe, seven-equation coarse LU-SGS, INTERT)."""
    from finflo_b200 import case
    from oracle.oracle import OracleMG
    lv_g, prms, fs = case.bump_case_mg(*dims, nlev=nlev, **SST)
    lv_c, _, _ = case.bump_case_mg(*dims, nlev=nlev, **SST)
    om = OracleMG(lv_c, prms)
    om.start()
    g = GpuSolver(0)
    bid = g.add_levels(lv_g, prms)
    for b in range(len(lv_g)):
        g.upload(bid + b)
    g.start(bid)
    n = 12
    hist = g.cycles(n, bid, icycle0=1, use_graph=True)
    ref = np.array([om.cycle(i + 1)[0] for i in range(n)])
    hist_close(hist[:, :5], ref, 1e-7)
    d = g.download(bid, ["TEMP", "U", "V", "RK", "REPS"])
    for nme in d:
        a = interior(lv_g[0], d[nme]); b = interior(lv_c[0], lv_c[0].arrays[nme])
        rel = np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-300)
        assert rel <= 1e-9, (nme, rel)
    g.close()
