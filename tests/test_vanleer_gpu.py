"""Van Leer flux-vector splitting (IFLUX=0, FLUXVL base3c.f:1733) on the
sm_100a path against the oracle: the residual per cell and whole cycles."""
import numpy as np
import pytest

from finflo_b200.gpu import GpuSolver
from oracle.oracle import Oracle
from tests.util import hist_close, flux_scale, interior, make_pair

pytestmark = pytest.mark.gpu

RES = ("DRO", "DM", "DN", "DW", "DE")


def _setup(dims=(17, 9, 9)):
    bg, bc, prm, fs = make_pair(*dims)
    prm.vanleer = 1
    o = Oracle(bc, prm)
    o.start()
    g = GpuSolver(0)
    bid = g.add_block(bg, prm)
    g.upload(bid)
    g.start(bid)
    return g, bid, bg, o, bc, prm


@pytest.mark.parametrize("dims", [(17, 9, 9), (33, 17, 9)])
def test_vanleer_residual(gpu_lib, dims):
    g, bid, bg, o, bc, prm = _setup(dims)
    o.statim(); o.adjuin(); o.residu(1, 1)
    g.residu(bid, 1, 1)
    g.sync()
    d = g.download(bid, list(RES))
    S = flux_scale(o, bc)
    for n in RES:
        ref = interior(bc, bc.arrays[n]); got = interior(bg, d[n])
        err = (np.abs(got - ref) / (np.maximum(np.abs(ref), S[n]) + 1e-300)).max()
        assert err <= 1e-12, (n, err)
    g.close()


def test_vanleer_cycles_match_oracle(gpu_lib):
    g, bid, bg, o, bc, prm = _setup()
    n = 30
    hist = g.cycles(n, bid, icycle0=1, use_graph=True)
    ref = np.array([o.cycle(i + 1)[0] for i in range(n)])
    hist_close(hist[:, :5], ref, 1e-8)
    d = g.download(bid, ["TEMP", "U", "V", "W", "PDIFF"])
    for nme in d:
        a = interior(bg, d[nme]); b = interior(bc, bc.arrays[nme])
        rel = np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-300)
        assert rel <= 1e-10, (nme, rel)
    g.close()
