"""Block set-up on the device (ff_block_metrics, ff_wall_distance) against
the host construction in finflo_b200/grid.py and case.py."""
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
def test_device_metrics_match_host(gpu_lib, kind):
    blk = case.bump_case(33, 17, 17)[0] if kind == "bump" else _warped_block()
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
        # unit-normal components on the scale of 1 (a component that is zero
        # on the host, e.g. the z part of a j face of an extruded grid, comes
        # out at rounding level with fused multiply-adds); the rest relative
        # to the array's largest magnitude
        scale = 1.0 if n.endswith(("XA", "YA", "ZA")) else np.abs(ref[n]).max()
        err = np.abs(d[n] - ref[n]).max() / scale
        assert err <= 1e-12, (n, err)
    g.close()


def test_device_multigrid_metrics_match_host(gpu_lib):
    """Three levels: the fine cells with 8 ghost layers, lumped twice."""
    levels, prms, fs = case.bump_case_mg(33, 17, 17, nlev=3)
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
            scale = 1.0 if n.endswith(("XA", "YA", "ZA")) else np.abs(ref[q][n]).max()
            err = np.abs(d[n] - ref[q][n]).max() / scale
            assert err <= 1e-12, (q, n, err)
    g.close()


def test_device_setup_runs_like_host_setup(gpu_lib):
    """The eight-block SST bump with two levels per block, set up on the
    host and on the device: the same residual history over 10 multi-block
    V-cycles (the two set-ups differ at rounding level in the metrics and by
    the host search's 1e-11 in DISTW)."""
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
                for q in range(2):
                    g.wall_distance(bid + q, out[3])
        g.start_all()
        hists.append(g.cycles_all(10, icycle0=1, use_graph=True)[:, :5])
        g.close()
    np.testing.assert_allclose(hists[1], hists[0], rtol=1e-6)


def _brute_force_distance(q, T):
    best = np.full(len(q), np.inf)
    for t in T:
        a, b, c = (np.broadcast_to(t[3 * m:3 * m + 3], q.shape) for m in range(3))
        np.minimum(best, case._closest_on_triangles(q, a, b, c), out=best)
    return best


def test_device_wall_distance(gpu_lib):
    """Exact distance to every wall triangle: against a host brute force, and
    never above the host's nearest-candidate search."""
    blk, prm, fs = case.bump_case(17, 9, 9, turbulence="sst", reynolds=1e6, mach=0.6, h1=1e-4)
    T = case.wall_triangles(blk)
    assert len(T) > 0
    q = np.stack([blk.arrays["XC"], blk.arrays["YC"], blk.arrays["ZC"]], axis=1)
    exact = _brute_force_distance(q, T)
    host = blk.arrays["DISTW"].copy()
    g = GpuSolver(0)
    bid = g.add_block(blk, prm)
    g.upload(bid)
    g.wall_distance(bid, T)
    d = g.download(bid, ["DISTW"])["DISTW"]
    np.testing.assert_allclose(d, exact, rtol=1e-12, atol=1e-15)
    assert (d <= host * (1 + 1e-12) + 1e-15).all()
    g.close()
