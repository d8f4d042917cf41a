"""Block set-up on the device (ff_block_metrics, ff_block_metrics_levels,
ff_wall_distance): the reference's construction (GRIDEX, AREVC1, D1D2D3,
LUMPA1, LUMPVS, PICK_XYZ, WALL_DIST, LUMP_DIST), written with
non-contracted arithmetic, equals the host set-up (finflo_b200/grid.py,
case.py) to the bit -- and through it the oracle's restatement
(tests/test_grid_setup_cpu.py)."""
import numpy as np
import pytest

from finflo_b200 import case, grid
from finflo_b200.gpu import GpuSolver

pytestmark = pytest.mark.gpu


def _warped_block():
    """A box with every interior node moved, so that no face is planar."""
    X, Y, Z = grid.box_nodes(np.linspace(0, 1, 21), np.linspace(0, 0.5, 11), np.linspace(0, 0.3, 7))
    rng = np.random.default_rng(3)
    for A, h in ((X, 0.05), (Y, 0.05), (Z, 0.05)):
        A[1:-1, 1:-1, 1:-1] += h * 0.3 * rng.uniform(-1, 1, A[1:-1, 1:-1, 1:-1].shape)
    fs = case.FlowConditions().freestream()
    return case.new_block(X, Y, Z, case.channel_patches(20, 10, 6, fs))


@pytest.mark.parametrize("kind", ["bump", "warped"])
def test_device_metrics_equal_host(gpu_lib, kind):
    blk = case.bump_case(33, 17, 17, span_amp=0.5, zlen=1.0)[0] if kind == "bump" else _warped_block()
    prm = case.make_params(case.FlowConditions(), blk.dims)
    ref = {n: blk.arrays[n].copy() for n in grid.METRIC_NAMES}
    for n in grid.METRIC_NAMES:
        blk.arrays[n][:] = 0.0
    g = GpuSolver(0)
    bid = g.add_block(blk, prm)
    g.upload(bid)
    g.block_metrics(bid, *blk.nodes)
    d = g.download(bid, list(grid.METRIC_NAMES))
    for n in grid.METRIC_NAMES:
        np.testing.assert_array_equal(d[n], ref[n], err_msg=n)
    g.close()


def test_device_multigrid_metrics_equal_host(gpu_lib):
    """Three levels: the fine cells with 8 ghost layers, lumped twice."""
    levels, prms, fs = case.bump_case_mg(33, 17, 17, nlev=3, span_amp=0.5, zlen=1.0)
    ref = [{n: lv.arrays[n].copy() for n in grid.METRIC_NAMES} for lv in levels]
    for lv in levels:
        for n in grid.METRIC_NAMES:
            lv.arrays[n][:] = 0.0
    g = GpuSolver(0)
    bid = g.add_levels(levels, prms)
    for q in range(len(levels)):
        g.upload(bid + q)
    g.block_metrics_levels(bid, 3, *levels[0].nodes)
    for q in range(len(levels)):
        d = g.download(bid + q, list(grid.METRIC_NAMES))
        for n in grid.METRIC_NAMES:
            np.testing.assert_array_equal(d[n], ref[q][n], err_msg=f"level {q + 1} {n}")
    g.close()


def test_device_wall_distance_equals_host(gpu_lib):
    """DISTW of all three levels (every cell of each, the coarse interior
    cells lumped) from the block's own wall points."""
    levels, prms, fs = case.bump_case_mg(33, 17, 17, nlev=3, turbulence="sst", reynolds=1e6, mach=0.6, h1=1e-4)
    ref = [lv.arrays["DISTW"].copy() for lv in levels]
    pts = case.wall_points(levels[0].nodes, levels[0].patches)
    assert len(pts) > 0
    g = GpuSolver(0)
    bid = g.add_levels(levels, prms)
    for q, lv in enumerate(levels):
        lv.arrays["DISTW"][:] = 0.0
        g.upload(bid + q)
    g.wall_distance(bid, pts)
    for q in range(len(levels)):
        d = g.download(bid + q, ["DISTW"])["DISTW"]
        np.testing.assert_array_equal(d, ref[q], err_msg=f"level {q + 1}")
    g.close()


def test_device_setup_runs_like_host_setup(gpu_lib):
    """The eight-block SST bump with two levels per block, set up on the
    host and on the device: identical set-up, identical residual history
    over 10 multi-block V-cycles."""
    kw = dict(cells=(40, 16, 16), nb=(2, 2, 2), nlev=2, reynolds=1e6, mach=0.6, h1=1e-4, cfl=1.0, cfll=1.0,
              lusgs_fp32=False, coarse_fp32=False, turbulence="sst")
    hists = []
    for dev in (False, True):
        out = case.bump_multiblock_case(**kw, device_setup=dev)
        bl, bp = out[0], out[1]
        g = GpuSolver(0)
        ids = g.add_multiblock(bl, bp)
        for bid in range(len(g.blocks)):
            g.upload(bid)
        if dev:
            for k, bid in enumerate(ids):
                g.block_metrics_levels(bid, 2, *bl[k][0].nodes)
                g.wall_distance(bid, out[3])
        g.start_all()
        hists.append(g.cycles_all(10, icycle0=1, use_graph=True)[:, :5])
        g.close()
    np.testing.assert_allclose(hists[1], hists[0], rtol=1e-12)
