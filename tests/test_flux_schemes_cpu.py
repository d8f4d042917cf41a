"""CPU tests of the IFLUX schemes besides Roe in their k-omega SST form
(FLUXKT base3c.f:4403 and FLUCUSP base3c.f:5133, called by RESIKE
res3c.f:7017-7036), and of the host's scheme checks:

* a uniform state: the seven-equation residual of KT and H-CUSP equals
  Roe's (the fluxes of a uniform state are exact in every scheme, the
  k-omega sources are the same);
* SST cycles on the bump channel: finite, the density residual falls;
* KT's wall face takes the pressure difference (YP4 = 1, base3c.f:6311):
  a uniform state's wall rows match Roe's."""
import numpy as np
import pytest

from finflo_b200 import case, grid
from oracle.oracle import Oracle
from tests.util import flux_scale, interior, momentum_floor

SST = dict(turbulence="sst", reynolds=1e6, mach=0.5, h1=1e-4)
RES7 = ("DRO", "DM", "DN", "DW", "DE", "DRK", "DEPS")


def _uniform_sst(flux):
    blk, prm, fs = case.bump_case(17, 9, 9, amp=0.0, noise=0.0, **SST)
    for pa in blk.patches:   # slip walls: the free stream is a solution
        if pa.ityp == grid.BC_SOL:
            pa.ityp = grid.BC_MIR
    prm.flux = case.FLUX[flux]
    o = Oracle(blk, prm)
    o.start()
    o.statim()
    o.turbeq()
    o.adjuin()
    o.residu_sst(1)
    return {n: interior(blk, blk.arrays[n]).copy() for n in RES7}, fs


@pytest.mark.parametrize("flux", ["kt", "hcusp"])
def test_uniform_state_residual_equals_roe(flux):
    ref, fs = _uniform_sst("roe")
    got, _ = _uniform_sst(flux)
    # per unit volume on cells of size ~1/16: flux scale * 16
    scale = {"DRO": fs["rho"] * fs["u"], "DM": fs["p"], "DN": fs["p"], "DW": fs["p"], "DE": fs["p"] * fs["u"] * 3.5}
    for n in RES7:
        s = 16 * scale[n] if n in scale else np.abs(ref[n]).max()
        assert np.abs(got[n] - ref[n]).max() <= 1e-10 * s, n


@pytest.mark.parametrize("flux", ["kt", "hcusp"])
def test_sst_cycles_fall(flux):
    blk, prm, fs = case.bump_case(17, 9, 9, **SST)
    prm.flux = case.FLUX[flux]
    o = Oracle(blk, prm)
    o.start()
    r = np.array([o.cycle(i + 1)[0] for i in range(60)])
    assert np.isfinite(r).all()
    assert r[-1, 0] < 0.05 * r[0, 0], r[-1, 0] / r[0, 0]


def test_kt_wall_takes_the_pressure_difference():
    """A uniform state on a flat no-slip channel: KT's wall rows get the same
    residual as Roe's.  KT's interior faces carry PDIFF and Roe's P, so this
    holds only because the wall face takes PDIFF for KT and P for Roe (YP1,
    YP4 base3c.f:6304-6315); a KT wall on P would leave FRSPRE * A / VOL."""
    blk, prm, fs = case.bump_case(9, 5, 5, amp=0.0, noise=0.0)
    out = {}
    for flux in ("roe", "kt"):
        b2, p2, _ = case.bump_case(9, 5, 5, amp=0.0, noise=0.0)
        p2.flux = case.FLUX[flux]
        o = Oracle(b2, p2)
        o.start()
        o.statim()
        o.adjuin()
        o.residu(1, 1)
        out[flux] = {n: interior(b2, b2.arrays[n]).copy() for n in ("DRO", "DN")}
    d = out["roe"]["DN"] - out["kt"]["DN"]   # per unit volume; FRSPRE * A / VOL ~ 1e3 * p here
    assert np.abs(d[:, [0, -1], :]).max() <= 1e-9 * fs["p"]
    np.testing.assert_allclose(out["roe"]["DRO"], out["kt"]["DRO"], rtol=0, atol=1e-9 * fs["rho"] * fs["u"])


def _residual(blk, prm, scale=False):
    o = Oracle(blk, prm)
    o.start()
    o.statim()
    o.adjuin()
    o.residu(1, 1)
    r = {n: interior(blk, blk.arrays[n]).copy() for n in RES7[:5]}
    return (r, flux_scale(o, blk)) if scale else r


@pytest.mark.parametrize("flux", ["roe", "kt", "hcusp"])
def test_xxtraa_equals_xxtrap_on_a_uniform_grid(flux):
    """XXTRAA (XXTRAL, base3c.f:1444) divides the differences by the centre
    distances and multiplies by the half extents: on equal cells that is
    XXTRAP's 1/4, so the unlimited (INTER = -3) residuals agree to 1e-10 of
    the cells' flux sums: XXTRAA adds EPS = 1e-10 to the centre distances
    (~0.2 here), a 5e-10 relative change of the extrapolation term.  (The
    van Albada limiter's EPS goes onto squared differences in XXTRAP and
    squared slopes in XXTRAA, so limited ones part where the differences
    are that small.)  On the stretched bump grid they differ."""
    out = []
    for xx in (0, 1):
        blk, prm, fs = case.bump_case(17, 9, 9, amp=0.0, h1=0.2, inter=-3)   # h1 above 1/8: uniform in y
        prm.flux, prm.xxtral = case.FLUX[flux], xx
        out.append(_residual(blk, prm, scale=True))
    (r0, S), (r1, _) = out
    S = momentum_floor(S)
    for n in r0:   # per cell, against the sum of its face fluxes' magnitudes
        assert (np.abs(r1[n] - r0[n]) / (np.maximum(np.abs(r0[n]), S[n]) + 1e-300)).max() <= 1e-10, n
    diff = []
    for xx in (0, 1):
        blk, prm, fs = case.bump_case(17, 9, 9)
        prm.flux, prm.xxtral = case.FLUX[flux], xx
        diff.append(_residual(blk, prm)["DRO"])
    assert np.abs(diff[1] - diff[0]).max() > 1e-6 * np.abs(diff[0]).max()


@pytest.mark.parametrize("flux", ["roe", "kt", "hcusp"])
def test_xxtral_cycles_fall(flux):
    blk, prm, fs = case.bump_case(17, 9, 9)
    prm.flux, prm.xxtral = case.FLUX[flux], 1
    o = Oracle(blk, prm)
    o.start()
    r = np.array([o.cycle(i + 1)[0][0] for i in range(60)])
    assert np.isfinite(r).all()
    assert r[-1] < 0.01 * r[0]


@pytest.mark.parametrize("sst", [False, True])
def test_jameson_dissipation_cycles(sst):
    """JAMESON (base3c.f:2827; RJK2 = 1/2, RJK4 = 1/64) on Roe's flux of the
    finest level: the residual of a uniform state stays Roe's (the
    differences vanish), the cycles converge, and the dissipation changes
    the residual of a disturbed state."""
    kw = dict(turbulence="sst", reynolds=1e6, mach=0.5, h1=1e-4) if sst else {}
    base, fs = None, None
    out = []
    for rj in ((0.0, 0.0), (0.5, 1.0 / 64)):
        blk, prm, fs = case.bump_case(17, 9, 9, **kw)
        prm.rjk2, prm.rjk4 = rj
        o = Oracle(blk, prm)
        o.start()
        r = np.array([o.cycle(i + 1)[0][0] for i in range(60)])
        assert np.isfinite(r).all()
        assert r[-1] < 0.01 * r[0]
        out.append(r)
    assert abs(out[1][1] - out[0][1]) > 1e-6 * out[0][1]


def test_jameson_keeps_the_free_stream():
    """A uniform laminar state on the flat slip-wall channel: the residual
    with JAMESON's dissipation is Roe's (every difference it takes is zero;
    SCALEJ is not).  (In the k-omega form OUTLET's ghost E carries rho*k
    once more than the interior's, so its last cells see a jump in E.)"""
    out = []
    for rj in ((0.0, 0.0), (0.5, 1.0 / 64)):
        blk, prm, fs = case.bump_case(17, 9, 9, amp=0.0, noise=0.0)
        for pa in blk.patches:
            if pa.ityp == grid.BC_SOL:
                pa.ityp = grid.BC_MIR
        prm.idi1 = prm.idi2 = prm.idi3 = 0
        prm.rjk2, prm.rjk4 = rj
        r, S = _residual(blk, prm, scale=True)
        out.append((r, S))
        if rj[0] > 0:
            assert np.abs(blk.arrays["SCALEJ"]).max() > 0
    (r0, S), (r1, _) = out
    S = momentum_floor(S)
    for n in r0:
        assert (np.abs(r1[n] - r0[n]) / (np.maximum(np.abs(r0[n]), S[n]) + 1e-300)).max() <= 1e-12, n
