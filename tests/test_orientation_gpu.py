"""1:1 patches in every orientation on the device: k_connec and the halo
pack read the donor cells through the same ICON(14) mapping as the
oracle's CONNEC (the 24 index-axis rotations of tests/test_orientation_cpu),
and the multi-block cycle of the turned pair follows the oracle's."""
import numpy as np
import pytest

from finflo_b200 import case
from finflo_b200.gpu import GpuSolver
from oracle.oracle import OracleMB
from tests.test_orientation_cpu import _field, _pair, rotations
from tests.util import hist_close, interior

pytestmark = pytest.mark.gpu


def _setup(rot):
    perm, flips = rotations()[rot]
    out = []
    for _ in range(2):
        A, B = _pair(perm, flips)
        fc = case.FlowConditions(mach=0.3, reynolds=1e4)
        fs = fc.freestream()
        prms = []
        for n, blk in enumerate((A, B)):
            case.init_freestream(blk, fs, noise=1e-2, seed=n)
            blk.arrays["TEMP"][:] *= 1.0 + 1e-3 * _field(blk)
            prms.append(case.make_params(fc, blk.dims, inter=1))
        out.append(((A, B), prms))
    return out


@pytest.mark.parametrize("rot", range(24))
def test_boundi_of_a_turned_pair_matches_oracle(gpu_lib, rot):
    (bg, pg), (bc, pc) = _setup(rot)
    om = OracleMB(list(bc), pc)
    om.boundi()
    g = GpuSolver(0)
    for b, p in zip(bg, pg):
        g.upload(g.add_block(b, p))
    g.boundi_all()
    g.sync()
    for bid in range(2):
        d = g.download(bid, ["TEMP", "U", "V", "W", "P", "PDIFF", "E"])
        for n, a in d.items():
            np.testing.assert_allclose(a, bc[bid].arrays[n], rtol=1e-13, atol=0, err_msg=f"block {bid} {n}")
    g.close()


@pytest.mark.parametrize("rot", [0, 5, 11, 17])
def test_cycles_of_a_turned_pair_match_oracle(gpu_lib, rot):
    (bg, pg), (bc, pc) = _setup(rot)
    om = OracleMB(list(bc), pc)
    om.start()
    g = GpuSolver(0)
    for b, p in zip(bg, pg):
        g.upload(g.add_block(b, p))
    g.start_all()
    hist = g.cycles_all(3, icycle0=1, use_graph=False)
    ref = np.array([om.cycle(i + 1)[0] for i in range(3)])
    hist_close(hist[:, :5], ref, 1e-9)
    for bid in range(2):
        d = g.download(bid, ["TEMP", "U", "V", "W"])
        for n, a in d.items():
            x, y = interior(bg[bid], a), interior(bc[bid], bc[bid].arrays[n])
            scale = np.linalg.norm(y) + np.linalg.norm(interior(bc[bid], bc[bid].arrays["U"]))
            assert np.linalg.norm(x - y) / scale <= 1e-11, (bid, n)
    g.close()
