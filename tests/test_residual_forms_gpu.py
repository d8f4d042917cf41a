"""Every residual form the autotuner chooses from -- tile shapes 32x4x4,
16x8x4, 8x8x8 cells, each with the face stencils read from global memory
or staged in shared memory -- gives the same residual to rounding (1e-14;
each kernel instantiation forms its own fused multiply-adds), and that
residual matches the oracle's (1e-12 of max(|R|, S) per cell).  The
block sizes are not multiples of the tiles, so partial tiles and the
stencil halo at the block's ghost layers are covered."""
import numpy as np
import pytest

from finflo_b200.gpu import GpuSolver
from oracle.oracle import Oracle
from tests.util import flux_scale, flux_scale_sst, interior, make_pair

pytestmark = pytest.mark.gpu

RES5 = ("DRO", "DM", "DN", "DW", "DE")
RES7 = RES5 + ("DRK", "DEPS")
SST = dict(turbulence="sst", reynolds=1e6, mach=0.6, h1=1e-4)


def _residual(form, sst, dims, monkeypatch):
    monkeypatch.setenv("FINFLO_RES_SHAPE", str(form))
    bg, bc, prm, fs = make_pair(*dims, **(SST if sst else {}))
    o = Oracle(bc, prm)
    o.start()
    g = GpuSolver(0)
    bid = g.add_block(bg, prm)
    g.upload(bid)
    g.start(bid)
    g.cycles(4, bid, icycle0=1, use_graph=False)     # the autotuner takes the fixed form
    assert g.residual_shape(bid) == ("32x4x4", "16x8x4", "8x8x8", "32x4x4 staged", "16x8x4 staged",
                                     "8x8x8 staged")[form]
    d = g.download(bid)
    for n, a in d.items():
        bc.arrays[n][:] = a
    names = RES7 if sst else RES5
    if sst:
        o.statim(); o.turbeq(); o.residu_sst(5)
    else:
        o.statim(); o.adjuin(); o.residu(1, 5)
    g.statim(bid)
    g.residu(bid, 1, 5)
    g.sync()
    got = g.download(bid, list(names))
    S = flux_scale_sst(o, bc) if sst else flux_scale(o, bc)
    for n in names:
        ref, x = interior(bc, bc.arrays[n]), interior(bg, got[n])
        err = (np.abs(x - ref) / (np.maximum(np.abs(ref), S[n]) + 1e-300)).max()
        assert err <= 1e-12, (form, n, err)
    g.close()
    return got


@pytest.mark.parametrize("sst", [False, True])
def test_residual_forms_agree_and_match_oracle(gpu_lib, sst, monkeypatch):
    dims = (38, 20, 11)      # 37 x 19 x 10 cells
    res = [_residual(f, sst, dims, monkeypatch) for f in range(6)]
    for f in range(1, 6):
        for n in res[0]:   # rounding-level: each instantiation contracts its own multiply-adds
            scale = np.abs(res[0][n]).max()
            np.testing.assert_allclose(res[f][n], res[0][n], rtol=1e-14, atol=1e-14 * scale,
                                       err_msg=f"form {f} {n}")
