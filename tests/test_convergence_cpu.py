"""CPU tests: convergence of the restated LU-SGS cycle on stretched grids.

PREDGS (imps4.f:1460-1466) shifts the i-direction products of a hyperplane
down by one index starting at IALKU, so the row-JMAX cell of the next
hyperplane never receives the i+1 product (its source index IALKU-1 is never
written).  On stretched grids at the reference's default CFL this makes the
lower sweep inconsistent with the diagonal and the iteration grows instead of
converging; ``ff_params.predgs_full`` keeps that coupling.  The converged
answer does not depend on the implicit operator (the fixed point is R(U) = 0),
so the switch changes only the path to it.
"""
import numpy as np

from finflo_b200 import case, grid
from oracle.oracle import Oracle


def _flat_slip_channel(predgs_full, ncyc=2000):
    """Inviscid uniform flow in a flat channel with slip (MIR) walls on a
    y-stretched grid (first cell 0.01), unlimited kappa = 1/3 MUSCL at
    CFL 3, density noise 1e-2: the exact answer is the free stream."""
    blk, prm, fs = case.bump_case(33, 17, 5, amp=0.0, h1=0.01, inter=-3, noise=1e-2, cfl=3.0)
    for pa in blk.patches:
        if pa.ityp == grid.BC_SOL:
            pa.ityp = grid.BC_MIR
    prm.idi1 = prm.idi2 = prm.idi3 = 0
    prm.fullns = 0
    prm.predgs_full = predgs_full
    o = Oracle(blk, prm)
    o.start()
    return np.array([o.cycle(i + 1)[0][0] for i in range(ncyc)])


def test_predgs_full_row_converges_where_reference_sweep_grows():
    ref = _flat_slip_channel(0)
    full = _flat_slip_channel(1)
    # the first residual precedes any implicit stage; after it the paths part
    assert ref[0] == full[0]
    assert full[-1] < 1e-5 * full[0], full[-1] / full[0]
    assert ref[-1] > ref[0], ref[-1] / ref[0]


def test_predgs_full_changes_only_the_path():
    """One implicit stage: the increments differ, but only through the
    lower sweep; a zero right-hand side stays zero either way."""
    blk, prm, fs = case.bump_case(17, 9, 5)
    o = Oracle(blk, prm)
    o.start()
    o.statim(); o.adjuin(); o.residu(1, 1)
    rhs = {n: blk.arrays[n].copy() for n in ("DRO", "DM", "DN", "DW", "DE")}
    out = []
    for full in (0, 1):
        for n in rhs:
            blk.arrays[n][:] = rhs[n]
        prm.predgs_full = full
        o.imps(1)
        out.append({n: blk.arrays[n].copy() for n in rhs})
    d = max(np.abs(out[0][n] - out[1][n]).max() / np.abs(out[0][n]).max() for n in rhs)
    assert d > 1e-8
    for n in rhs:
        blk.arrays[n][:] = 0.0
    o.imps(1)
    assert all(np.abs(blk.arrays[n]).max() == 0.0 for n in rhs)
