"""A device run written to RSTART (WRITRS outp3.f:2042) and continued from it
on a fresh block (READRS outp3.f:1119, then the usual start-up) follows the
oracle's uninterrupted run."""
import numpy as np
import pytest

from finflo_b200 import fileio
from finflo_b200.gpu import GpuSolver
from oracle.oracle import Oracle
from tests.util import make_pair

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
    np.testing.assert_allclose(hist[:, :5], ref[10:], rtol=1e-8)
    g2.close()
