"""A device run written to RSTART (WRITRS outp3.f:2042) and continued from it
on a fresh block (READRS outp3.f:1119, then the usual start-up) follows the
oracle's uninterrupted run."""
import numpy as np
import pytest

from finflo_b200 import fileio
from finflo_b200.gpu import GpuSolver
from oracle.oracle import Oracle
from tests.util import hist_close, make_pair

pytestmark = pytest.mark.gpu

SST = dict(turbulence="sst", reynolds=1e6, mach=0.6, h1=1e-4)


@pytest.mark.parametrize("sst", [False, True])
def test_restart_continues_the_device_run(gpu_lib, tmp_path, sst):
    kw = SST if sst else {}
    bg, bc, prm, fs = make_pair(17, 9, 9, **kw)
    o = Oracle(bc, prm)
    o.start()
    ref = np.array([o.cycle(i + 1)[0] for i in range(15)])

    g = GpuSolver(0)
    bid = g.add_block(bg, prm)
    g.upload(bid)
    g.start(bid)
    g.cycles(10, bid, icycle0=1)
    names = [n for n in dict.fromkeys(fileio.RESTART_FIELDS) if n in bg.arrays]
    path = tmp_path / "RSTART"
    fileio.write_restart(path, [g.download(bid, names)])
    g.close()

    bg2, _, prm2, _ = make_pair(17, 9, 9, **kw)
    time2, got = fileio.read_restart(path, [bg2.ntot])
    assert not time2
    fileio.load_restart_vars(bg2, got[0])
    g2 = GpuSolver(0)
    bid2 = g2.add_block(bg2, prm2)
    g2.upload(bid2)
    g2.start(bid2)
    hist = g2.cycles(5, bid2, icycle0=11)
    hist_close(hist[:, :5], ref[10:], 1e-8)
    g2.close()


def test_restart_continues_a_timel_device_run(gpu_lib, tmp_path):
    """Time-accurate device run: two physical steps, RSTART with the
    time-level records, a fresh device block read from it whose next step
    begins with NEWTIM; its third step follows the oracle's uninterrupted
    three steps."""
    inner, dt = 8, 2e-5
    bg, bc, prm, fs = make_pair(17, 9, 9)
    prm.timel, prm.dt = 1, dt
    o = Oracle(bc, prm)
    o.start()
    o.time_levels(0)
    ref = []
    for s in range(3):
        if s:
            o.time_levels(1)
        ref += [o.cycle(i + 1)[0] for i in range(inner)]

    g = GpuSolver(0)
    bid = g.add_block(bg, prm)
    g.upload(bid)
    g.start(bid)
    g.time_levels(bid, 0)
    for s in range(2):
        if s:
            g.time_levels(bid, 1)
        g.cycles(inner, bid, icycle0=1)
    names = [n for n in dict.fromkeys(fileio.RESTART_FIELDS + fileio.RESTART_TIME_FIELDS) if n in bg.arrays]
    path = tmp_path / "RSTART"
    fileio.write_restart(path, [g.download(bid, names)], timel=True)
    g.close()

    bg2, _, prm2, _ = make_pair(17, 9, 9)
    prm2.timel, prm2.dt = 1, dt
    time2, got = fileio.read_restart(path, [bg2.ntot], timel=True)
    assert time2
    fileio.load_restart_vars(bg2, got[0])
    g2 = GpuSolver(0)
    bid2 = g2.add_block(bg2, prm2)
    g2.upload(bid2)
    g2.start(bid2)
    g2.time_levels(bid2, 1)   # NEWTIM: the file's level n becomes n-1, the state level n
    hist = g2.cycles(inner, bid2, icycle0=1)
    hist_close(hist[:, :5], np.array(ref[2 * inner:]), 1e-8)
    g2.close()
