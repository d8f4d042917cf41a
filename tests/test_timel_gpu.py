"""Time-accurate dual time stepping (TIMEL) on the sm_100a path against the
oracle: the residual with the time derivative, and whole physical steps
(STARTI, inner cycles, NEWTIM, inner cycles) for the laminar and the SST
equations."""
import numpy as np
import pytest

from finflo_b200.gpu import GpuSolver
from oracle.oracle import Oracle
from tests.util import interior, make_pair

pytestmark = pytest.mark.gpu

SST = dict(turbulence="sst", reynolds=1e6, mach=0.6, h1=1e-4)


def _setup(sst, dt):
    bg, bc, prm, fs = make_pair(17, 9, 9, **(SST if sst else {}))
    prm.timel, prm.dt = 1, dt
    o = Oracle(bc, prm)
    o.start()
    o.time_levels(0)
    g = GpuSolver(0)
    bid = g.add_block(bg, prm)
    g.upload(bid)
    g.start(bid)
    g.time_levels(bid, 0)
    return g, bid, bg, o, bc


@pytest.mark.parametrize("sst", [False, True])
def test_timel_physical_steps_match_oracle(gpu_lib, sst):
    """Three physical steps of 8 inner cycles: residual history (the time
    derivative included) and fields."""
    g, bid, bg, o, bc = _setup(sst, 5e-5)
    hist, ref = [], []
    for step in range(3):
        if step:
            o.time_levels(1)
            g.time_levels(bid, 1)
        hist.append(g.cycles(8, bid, icycle0=1, use_graph=bool(step % 2)))
        ref.append(np.array([o.cycle(i + 1)[0] for i in range(8)]))
    np.testing.assert_allclose(np.concatenate(hist)[:, :5], np.concatenate(ref), rtol=1e-8)
    names = ["TEMP", "U", "V", "W", "PDIFF"] + (["RK", "REPS"] if sst else [])
    d = g.download(bid, names + ["ROLE2", "ROLE3"])
    for n in names + ["ROLE2", "ROLE3"]:
        a = interior(bg, d[n]); b = interior(bc, bc.arrays[n])
        rel = np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-300)
        assert rel <= 1e-10, (n, rel)
    g.close()


def test_timel_residual_matches_oracle(gpu_lib):
    """One residual evaluation with old time levels that differ from the
    state: per cell within 1e-12 of the largest residual."""
    g, bid, bg, o, bc = _setup(False, 1e-5)
    for i in range(3):
        o.cycle(i + 1)
    g.cycles(3, bid, icycle0=1)
    o.time_levels(1)
    g.time_levels(bid, 1)
    o.cycle(4)
    g.cycles(1, bid, icycle0=4)
    o.statim(); o.adjuin(); o.residu(1, 5)
    g.residu(bid, 1, 5)
    g.sync()
    d = g.download(bid, ["DRO", "DM", "DN", "DW", "DE"])
    for n in d:
        ref = interior(bc, bc.arrays[n]); got = interior(bg, d[n])
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max(), n
    g.close()
