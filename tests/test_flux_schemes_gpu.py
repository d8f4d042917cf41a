"""The IFLUX schemes besides Roe (ff_params.flux) on the sm_100a path
against the oracle: van Leer FLUXVL (base3c.f:1733), WPS FLUXWP (1967), AUSM
FLUXAU (2201), Kurganov-Tadmor FLUXKT (4403) and H-CUSP FLUCUSP (5133).

* the laminar residual per cell (1e-12 of max(|R|, S)) of all five, and the
  k-omega SST residual of KT and H-CUSP, the two that RESIKE offers;
* whole cycles: residual histories and fields, single-grid laminar and SST,
  and a two-level V-cycle (the coarse level's first-order faces);
* the library refuses a laminar-only scheme on a k-omega block and an
  unknown scheme."""
import numpy as np
import pytest

from finflo_b200 import case, grid
from finflo_b200.gpu import FinfloGpuError, GpuSolver
from oracle.oracle import Oracle, OracleMG
from tests.util import hist_close, flux_scale, flux_scale_sst, interior, make_pair, momentum_floor

pytestmark = pytest.mark.gpu

RES = ("DRO", "DM", "DN", "DW", "DE")
RES7 = RES + ("DRK", "DEPS")
LAMINAR = ["vanleer", "wps", "ausm", "kt", "hcusp"]
SST = dict(turbulence="sst", reynolds=1e6, mach=0.6, h1=1e-4)


def _slip(blk, prm):
    """No-slip walls to slip (MIR) walls, inviscid: the case AUSM converges
    on (its momentum flux carries PDIFF, BOTSKE's wall P)."""
    for pa in blk.patches:
        if pa.ityp == grid.BC_SOL:
            pa.ityp = grid.BC_MIR
    prm.idi1 = prm.idi2 = prm.idi3 = 0
    prm.fullns = 0


def _setup(flux, dims=(17, 9, 9), **kw):
    bg, bc, prm, fs = make_pair(*dims, **kw)
    if flux == "ausm":
        _slip(bg, prm)
        _slip(bc, prm)
    prm.flux = case.FLUX[flux]
    o = Oracle(bc, prm)
    o.start()
    g = GpuSolver(0)
    bid = g.add_block(bg, prm)
    g.upload(bid)
    g.start(bid)
    return g, bid, bg, o, bc, prm


@pytest.mark.parametrize("dims", [(17, 9, 9), (33, 17, 9)])
@pytest.mark.parametrize("flux", LAMINAR)
def test_laminar_residual(gpu_lib, flux, dims):
    g, bid, bg, o, bc, prm = _setup(flux, dims)
    o.statim(); o.adjuin(); o.residu(1, 1)
    g.residu(bid, 1, 1)
    g.sync()
    d = g.download(bid, list(RES))
    S = momentum_floor(flux_scale(o, bc))
    for n in RES:
        ref = interior(bc, bc.arrays[n]); got = interior(bg, d[n])
        err = (np.abs(got - ref) / (np.maximum(np.abs(ref), S[n]) + 1e-300)).max()
        assert err <= 1e-12, (flux, n, err)
    g.close()


@pytest.mark.parametrize("flux", LAMINAR)
def test_laminar_cycles_match_oracle(gpu_lib, flux):
    kw = dict(cfl=1.0) if flux == "ausm" else {}
    g, bid, bg, o, bc, prm = _setup(flux, **kw)
    n = 30
    hist = g.cycles(n, bid, icycle0=1, use_graph=True)
    ref = np.array([o.cycle(i + 1)[0] for i in range(n)])
    hist_close(hist[:, :5], ref, 1e-8)
    d = g.download(bid, ["TEMP", "U", "V", "W", "PDIFF"])
    for nme in d:
        a = interior(bg, d[nme]); b = interior(bc, bc.arrays[nme])
        rel = np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-300)
        assert rel <= 1e-10, (flux, nme, rel)
    g.close()


@pytest.mark.parametrize("flux", ["kt", "hcusp"])
def test_sst_residual(gpu_lib, flux):
    """RESIKE with FLUXKT / FLUCUSP after a few cycles (k, omega, mu_t
    varying): the seven residuals per cell within 1e-12 of max(|R|, S)."""
    g, bid, bg, o, bc, prm = _setup(flux, **SST)
    for i in range(5):
        o.cycle(i + 1)
    g.cycles(5, bid, icycle0=1, use_graph=False)
    d = g.download(bid)
    for n, a in d.items():
        bc.arrays[n][:] = a
    o.statim(); o.turbeq(); o.residu_sst(6)
    g.statim(bid); g.residu(bid, 1, 6)
    g.sync()
    got_all = g.download(bid, list(RES7))
    S = momentum_floor(flux_scale_sst(o, bc))
    for n in RES7:
        ref = interior(bc, bc.arrays[n]); got = interior(bg, got_all[n])
        err = (np.abs(got - ref) / (np.maximum(np.abs(ref), S[n]) + 1e-300)).max()
        assert err <= 1e-12, (flux, n, err)
    g.close()


@pytest.mark.parametrize("flux", ["kt", "hcusp"])
def test_sst_cycles_match_oracle(gpu_lib, flux):
    g, bid, bg, o, bc, prm = _setup(flux, **SST)
    n = 20
    hist = g.cycles(n, bid, icycle0=1, use_graph=True)
    ref = np.array([o.cycle(i + 1)[0] for i in range(n)])
    hist_close(hist[:, :5], ref, 1e-8)
    d = g.download(bid, ["TEMP", "U", "V", "PDIFF", "RK", "REPS"])
    for nme in d:
        a = interior(bg, d[nme]); b = interior(bc, bc.arrays[nme])
        rel = np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-300)
        assert rel <= 1e-9, (flux, nme, rel)
    g.close()


@pytest.mark.parametrize("flux", ["wps", "kt", "hcusp"])
def test_multigrid_cycles_match_oracle(gpu_lib, flux):
    """Two-level FAS V-cycles: the coarse level's faces in the same scheme
    at its own INTEM (first order, 55)."""
    lv_g, prms, fs = case.bump_case_mg(17, 9, 9, nlev=2)
    lv_c, _, _ = case.bump_case_mg(17, 9, 9, nlev=2)
    for q in prms:
        q.flux = case.FLUX[flux]
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
    d = g.download(bid, ["TEMP", "U", "V", "PDIFF"])
    for nme in d:
        a = interior(lv_g[0], d[nme]); b = interior(lv_c[0], lv_c[0].arrays[nme])
        rel = np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-300)
        assert rel <= 1e-9, (flux, nme, rel)
    g.close()


def test_scheme_checks(gpu_lib):
    blk, prm, fs = case.bump_case(9, 5, 5, **SST)
    g = GpuSolver(0)
    for flux in ("vanleer", "wps", "ausm"):
        prm.flux = case.FLUX[flux]
        with pytest.raises(FinfloGpuError, match="laminar only"):
            g.add_block(blk, prm)
    prm.flux = 5
    with pytest.raises(FinfloGpuError, match="unknown scheme"):
        g.add_block(blk, prm)
    for flux in ("kt", "hcusp", "roe"):
        prm.flux = case.FLUX[flux]
        g.add_block(blk, prm)
    g.close()


@pytest.mark.parametrize("flux", ["roe", "kt", "hcusp"])
@pytest.mark.parametrize("sst", [False, True])
def test_xxtral_residual(gpu_lib, flux, sst):
    """XXTRAL (XXTRAA base3c.f:1444, the MUSCL over the cells' extents) with
    Roe, KT and H-CUSP on the stretched bump grid, laminar and SST: the
    residual per cell within 1e-12 of max(|R|, S)."""
    g, bid, bg, o, bc, prm = _setup(flux, **(SST if sst else {}))
    prm.xxtral = 1
    g.set_params(bid, prm)
    if sst:
        o.statim(); o.turbeq(); o.residu_sst(1)
    else:
        o.statim(); o.adjuin(); o.residu(1, 1)
    g.residu(bid, 1, 1)
    g.sync()
    names = RES7 if sst else RES
    d = g.download(bid, list(names))
    S = momentum_floor(flux_scale_sst(o, bc) if sst else flux_scale(o, bc))
    for n in names:
        ref = interior(bc, bc.arrays[n]); got = interior(bg, d[n])
        err = (np.abs(got - ref) / (np.maximum(np.abs(ref), S[n]) + 1e-300)).max()
        assert err <= 1e-12, (flux, n, err)
    g.close()


@pytest.mark.parametrize("sst", [False, True])
def test_xxtral_cycles_match_oracle(gpu_lib, sst):
    g, bid, bg, o, bc, prm = _setup("roe", **(SST if sst else {}))
    prm.xxtral = 1
    g.set_params(bid, prm)
    n = 20
    hist = g.cycles(n, bid, icycle0=1, use_graph=True)
    ref = np.array([o.cycle(i + 1)[0] for i in range(n)])
    hist_close(hist[:, :5], ref, 1e-8)
    g.close()


@pytest.mark.parametrize("sst", [False, True])
def test_jameson_residual(gpu_lib, sst):
    """JAMESON's dissipation (RJK2 = 1/2, RJK4 = 1/64; SCALARD's SCALEJ) on
    Roe's flux: the residual per cell after a few cycles, and SCALEJ."""
    g, bid, bg, o, bc, prm = _setup("roe", **(SST if sst else {}))
    prm.rjk2, prm.rjk4 = 0.5, 1.0 / 64
    g.set_params(bid, prm)
    for i in range(3):
        o.cycle(i + 1)
    g.cycles(3, bid, icycle0=1, use_graph=False)
    d = g.download(bid)
    for n, a in d.items():
        bc.arrays[n][:] = a
    if sst:
        o.statim(); o.turbeq(); o.residu_sst(4)
        g.statim(bid); g.residu(bid, 1, 4)
    else:
        o.statim(); o.adjuin(); o.residu(1, 4)
        g.statim(bid); g.residu(bid, 1, 4)
    g.sync()
    names = RES7 if sst else RES
    got_all = g.download(bid, list(names) + ["SCALEJ"])
    a, b = interior(bg, got_all["SCALEJ"]), interior(bc, bc.arrays["SCALEJ"])
    assert np.abs(a - b).max() <= 1e-13 * np.abs(b).max()
    S = momentum_floor(flux_scale_sst(o, bc) if sst else flux_scale(o, bc))
    for n in names:
        ref = interior(bc, bc.arrays[n]); got = interior(bg, got_all[n])
        err = (np.abs(got - ref) / (np.maximum(np.abs(ref), S[n]) + 1e-300)).max()
        assert err <= 1e-12, (n, err)
    g.close()


@pytest.mark.parametrize("sst", [False, True])
def test_jameson_cycles_match_oracle(gpu_lib, sst):
    g, bid, bg, o, bc, prm = _setup("roe", **(SST if sst else {}))
    prm.rjk2, prm.rjk4 = 0.5, 1.0 / 64
    g.set_params(bid, prm)
    n = 20
    hist = g.cycles(n, bid, icycle0=1, use_graph=True)
    ref = np.array([o.cycle(i + 1)[0] for i in range(n)])
    hist_close(hist[:, :5], ref, 1e-8)
    g.close()
