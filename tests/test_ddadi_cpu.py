"""The oracle's DDADI implicit stage (LUSGS=0, IMPSWE imps3.f:578 with
PRED/DIAG/CORR imps4.f:671-971 and the k-omega forms): properties that hold
at any size, convergence of whole cycles, and the regression pin."""
import os

import numpy as np
import pytest

from finflo_b200 import case
from oracle.oracle import Oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RES5 = ("DRO", "DM", "DN", "DW", "DE")
RES7 = RES5 + ("DRK", "DEPS")
SST = dict(turbulence="sst", reynolds=1e6, mach=0.6, h1=1e-4)


def _primed(sst):
    """A block a few cycles in, with the residual turned into the primitive
    right-hand side that the line sweeps take (TIME3, LOCDT(K), COPR(KE))."""
    blk, prm, fs = case.bump_case(17, 9, 9, **(SST if sst else {}))
    prm.ddadi = 1
    o = Oracle(blk, prm)
    o.start()
    for i in range(3):
        o.cycle(i + 1)
    return blk, prm, o


@pytest.mark.parametrize("sst", [False, True])
def test_sweeps_are_linear_in_the_right_hand_side(sst):
    """For a fixed state the DDADI stage is a linear map of the increments:
    DDADI(2a - 3b) = 2 DDADI(a) - 3 DDADI(b) to rounding."""
    blk, prm, o = _primed(sst)
    names = RES7 if sst else RES5
    rng = np.random.default_rng(0)
    a = {n: rng.standard_normal(blk.arrays[n].shape) for n in names}
    b = {n: rng.standard_normal(blk.arrays[n].shape) for n in names}
    interior = np.zeros(blk.arrays["DRO"].shape, bool)
    interior.reshape(blk.kmax + 4, blk.jmax + 4, blk.imax + 4)[2:-2, 2:-2, 2:-2] = True

    def run(x):
        for n in names:
            blk.arrays[n][:] = np.where(interior, x[n], 0.0)
        o.ddadi()
        return {n: blk.arrays[n].copy() for n in names}

    ra, rb = run(a), run(b)
    rc = run({n: 2 * a[n] - 3 * b[n] for n in names})
    for n in names:
        ref = 2 * ra[n] - 3 * rb[n]
        assert np.abs(rc[n] - ref).max() <= 1e-12 * np.abs(ref).max(), n
        assert not rc[n][~interior].any(), n      # ghost increments stay zero


@pytest.mark.parametrize("sst", [False, True])
def test_ddadi_cycles_converge(sst):
    blk, prm, fs = case.bump_case(17, 9, 9, **(SST if sst else {}))
    prm.ddadi = 1
    o = Oracle(blk, prm)
    o.start()
    r = np.array([o.cycle(i + 1)[0][0] for i in range(60)])
    assert np.isfinite(r).all()
    assert r[-1] < 0.2 * r[0]


def test_ddadi_golden_history():
    """Regression pin of the oracle's DDADI path (tests/golden/make_golden.py)."""
    g = np.load(os.path.join(ROOT, "tests", "golden", "bump_17x9x9_ddadi.npz"))
    blk, prm, fs = case.bump_case(17, 9, 9)
    prm.ddadi = 1
    o = Oracle(blk, prm)
    o.start()
    hist = np.array([o.cycle(i + 1)[0] for i in range(10)])
    np.testing.assert_allclose(hist, g["hist10"], rtol=1e-11)
