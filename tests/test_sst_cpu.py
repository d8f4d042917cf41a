"""k-omega SST in the CPU oracle: set-up, limits and convergence."""
import numpy as np

from finflo_b200 import case
from oracle.oracle import Oracle


def test_sst_freestream_values():
    fc = case.FlowConditions(mach=0.6, reynolds=1e6)
    fs = fc.freestream()
    rk, re = case.sst_freestream(fs, tu=1e-3, mut_ratio=0.1)
    assert np.isclose(rk, 1.5 * fs["rho"] * (1e-3 * fs["u"]) ** 2)
    # mu_t = rho k / omega = 0.1 mu
    assert np.isclose((rk / fs["rho"]) / (re / fs["rho"]) * fs["rho"], 0.1 * fs["mu"])


def test_wall_distance_is_the_distance_to_the_walls():
    blk, prm, fs = case.bump_case(17, 9, 5, turbulence="sst", h1=1e-2)
    d = blk.interior("DISTW")
    y = blk.interior("YC")
    # first cell row above the flat part of the lower wall (x < 1)
    x = blk.interior("XC")
    flat = x[:, 0, :] < 0.9
    assert np.allclose(d[:, 0, :][flat], y[:, 0, :][flat], rtol=1e-6)
    assert (d > 0).all() and d.max() <= 0.5 + 1e-9


def test_sst_cycles_converge_and_respect_limits():
    blk, prm, fs = case.bump_case(33, 17, 9, turbulence="sst", reynolds=1e6, mach=0.6, h1=1e-4, noise=0.0)
    o = Oracle(blk, prm)
    o.start()
    h = np.sqrt(np.array([o.cycle(i + 1)[0][0] for i in range(150)]))
    assert np.isfinite(h).all()
    assert h[-1] < 0.05 * h[0]
    rk, re = blk.interior("RK"), blk.interior("REPS")
    assert rk.min() >= prm.rklim and re.min() >= prm.epslim
    mut = blk.interior("VIST") / blk.interior("VIS")
    assert mut.max() <= prm.turlim
    # k grows from the free-stream value in the boundary layers
    assert rk.max() > 5 * prm.rklim


def test_sst_multigrid_beats_single_grid():
    """The 3-level SST V-cycle reduces the density residual faster per cycle
    than the single-grid iteration on the same grid."""
    from oracle.oracle import OracleMG
    kw = dict(turbulence="sst", reynolds=1e6, mach=0.6, h1=1e-4, noise=0.0)
    lv, prms, fs = case.bump_case_mg(33, 17, 17, nlev=3, **kw)
    om = OracleMG(lv, prms)
    om.start()
    hm = np.sqrt(np.array([om.cycle(i + 1)[0][0] for i in range(80)]))
    b, p, _ = case.bump_case(33, 17, 17, **kw)
    o = Oracle(b, p)
    o.start()
    hs = np.sqrt(np.array([o.cycle(i + 1)[0][0] for i in range(80)]))
    assert np.isfinite(hm).all()
    assert hm[-1] / hm[0] < 0.5 * hs[-1] / hs[0]
    assert lv[0].interior("RK").min() >= prms[0].rklim
