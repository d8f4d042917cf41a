"""Time-accurate dual time stepping (TIMEL) in the oracle: TIMDER
res3c.f:3014 / TIMDKE res3c.f:3062, the dual time step of TIME3
(base3c.f:206-215), STARTI res3c.f:3175 and NEWTIM ns3c.f:9420."""
import numpy as np
import pytest

from finflo_b200 import case
from oracle.oracle import Oracle
from tests.util import interior

SST = dict(turbulence="sst", reynolds=1e6, mach=0.6, h1=1e-4)
Q5 = ("RO", "RM", "RN", "RW", "E")
Q7 = Q5 + ("RK", "REPS")
RES7 = ("DRO", "DM", "DN", "DW", "DE", "DRK", "DEPS")


def test_timder_is_second_order_backward_difference():
    """With the three time levels of Q(t) = a + b t + c t^2 at t = 0, -dt,
    -2dt the added term is -VOL dQ/dt(0) / VOL = -b exactly (BDF2 is exact for
    quadratics), on every interior cell and nowhere else."""
    blk, prm, fs = case.bump_case(9, 7, 5, **SST)
    prm.timel, prm.dt = 1, 0.25
    o = Oracle(blk, prm)
    rng = np.random.default_rng(1)
    a, bb, c = (rng.standard_normal(blk.arrays["RO"].shape) for _ in range(3))
    dt = prm.dt
    for q, q2, q3 in zip(Q7, [n + "LE2" if n != "REPS" else "EPSLE2" for n in Q7],
                         [n + "LE3" if n != "REPS" else "EPSLE3" for n in Q7]):
        blk.arrays[q][:] = a
        blk.arrays[q2][:] = a - bb * dt + c * dt * dt
        blk.arrays[q3][:] = a - 2 * bb * dt + 4 * c * dt * dt
    for n in RES7:
        blk.arrays[n][:] = 0.0
    o.L.orc_timder(o._b(), o._p(), 7)
    for n in RES7:
        np.testing.assert_allclose(interior(blk, blk.arrays[n]), interior(blk, -bb), rtol=1e-12, atol=1e-12)
        d = blk.arrays[n].reshape(blk.kmax + 4, blk.jmax + 4, blk.imax + 4).copy()
        d[2:-2, 2:-2, 2:-2] = 0.0
        assert not d.any()


@pytest.mark.parametrize("sst", [False, True])
def test_infinite_physical_step_is_the_steady_run(sst):
    """DT -> infinity: the dual time step equals the local step and the time
    derivative vanishes, so the cycles repeat the steady run."""
    kw = SST if sst else {}
    runs = []
    for timel in (0, 1):
        blk, prm, fs = case.bump_case(17, 9, 9, **kw)
        prm.timel, prm.dt = timel, 1e30
        o = Oracle(blk, prm)
        o.start()
        if timel:
            o.time_levels(0)
        runs.append(np.array([o.cycle(i + 1)[0] for i in range(12)]))
    np.testing.assert_allclose(runs[1], runs[0], rtol=1e-12)


def test_time_levels_startup_and_shift():
    blk, prm, fs = case.bump_case(9, 7, 5)
    prm.timel, prm.dt = 1, 1e-3
    o = Oracle(blk, prm)
    o.start()
    o.time_levels(0)
    for q in Q5:
        np.testing.assert_array_equal(blk.arrays[q + "LE2"], blk.arrays[q])
        np.testing.assert_array_equal(blk.arrays[q + "LE3"], blk.arrays[q])
    o.cycle(1)
    old = {q: blk.arrays[q + "LE2"].copy() for q in Q5}
    o.time_levels(1)
    for q in Q5:
        np.testing.assert_array_equal(interior(blk, blk.arrays[q + "LE3"]), interior(blk, old[q]))
        np.testing.assert_array_equal(interior(blk, blk.arrays[q + "LE2"]), interior(blk, blk.arrays[q]))


def test_physical_steps_converge_inside_each_step():
    """Two physical steps of 25 inner cycles each: inside every step the
    inner (pseudo-time) iterations drive the residual down."""
    blk, prm, fs = case.bump_case(17, 9, 9)
    prm.timel, prm.dt = 1, 2e-5
    o = Oracle(blk, prm)
    o.start()
    o.time_levels(0)
    for step in range(2):
        if step:
            o.time_levels(1)
        r = np.array([o.cycle(i + 1)[0][0] for i in range(25)])
        assert np.isfinite(r).all()
        assert r[-1] < 1e-2 * r[0], (step, r[0], r[-1])
