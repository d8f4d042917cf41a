"""FP32 coarse levels (ff_params.res_fp32 on levels 2+ with lusgs_fp32): the
coarse levels' face fluxes and implicit stage in FP32, the fine level's
residual, every update, the transfers and the norms in FP64.

* one coarse-level residual in FP32 against the same residual in FP64
  (which tests/test_stages_gpu.py holds to the oracle): FP32 rounding;
* a laminar two-level case run to convergence (12 decades of the density
  residual's sum of squares) with the FP32 coarse level: the converged
  fine fields equal the FP64 oracle's to 1e-8.  The coarse levels only
  steer the path: at the fine fixed point the FAS forcing makes the
  coarse correction vanish whatever the coarse arithmetic."""
import numpy as np
import pytest

from finflo_b200 import case
from finflo_b200.gpu import GpuSolver
from oracle.oracle import OracleMG
from tests.util import interior

pytestmark = pytest.mark.gpu

RES5 = ["DRO", "DM", "DN", "DW", "DE"]
RES7 = RES5 + ["DRK", "DEPS"]
SST = dict(turbulence="sst", reynolds=1e6, mach=0.6, h1=1e-4)


@pytest.mark.parametrize("sst", [False, True])
def test_coarse_residual_in_fp32(gpu_lib, sst):
    out = {}
    for fp32 in (0, 1):
        levels, prms, fs = case.bump_case_mg(33, 17, 17, nlev=2, **(SST if sst else {}))
        prms[1].res_fp32 = fp32
        g = GpuSolver(0)
        bid = g.add_levels(levels, prms)
        for q in range(2):
            g.upload(bid + q)
        g.start(bid)
        g.cycles(3, bid, icycle0=1, use_graph=False)
        g.statim(bid + 1)
        g.residu(bid + 1, 2, 1)
        g.sync()
        out[fp32] = g.download(bid + 1, RES7 if sst else RES5)
        g.close()
    for n in out[0]:
        ref, got = out[0][n], out[1][n]
        err = np.abs(got - ref).max() / np.abs(ref).max()
        assert 0.0 < err <= 2e-5, (n, err)   # FP32 rounding: not bitwise, not more


LAM = dict(amp=0.05, inter=1, cfl=2.0, cfll=2.0)
LAM_CYC = 5000


def test_fp32_coarse_level_converges_to_the_fp64_oracle_fields(gpu_lib):
    lc, pc, _ = case.bump_case_mg(33, 17, 9, nlev=2, **LAM)
    for q in pc:
        q.predgs_full = 1
    om = OracleMG(lc, pc)
    om.start()
    href = np.array([om.cycle(i + 1)[0][0] for i in range(LAM_CYC)])
    lg, pg, _ = case.bump_case_mg(33, 17, 9, nlev=2, coarse_fp32=True, coarse_res_fp32=True, **LAM)
    for q in pg:
        q.predgs_full = 1
    g = GpuSolver(0)
    bid = g.add_levels(lg, pg)
    for q in range(2):
        g.upload(bid + q)
    g.start(bid)
    h = g.cycles(LAM_CYC, bid, icycle0=1)[:, 0]
    assert np.log10(href[0] / href[-1]) >= 12.0
    assert np.log10(h[0] / h[-1]) >= 12.0
    names = ["TEMP", "U", "V", "W", "PDIFF", "RO", "E"]
    d = g.download(bid, names)
    scale_u = np.linalg.norm(interior(lc[0], lc[0].arrays["U"]))
    for n in names:
        a, b = interior(lg[0], d[n]), interior(lc[0], lc[0].arrays[n])
        rel = np.linalg.norm(a - b) / (scale_u if n == "W" else np.linalg.norm(b))
        assert rel <= 1e-8, (n, rel)
    g.close()
