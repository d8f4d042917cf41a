"""Parity of the sm_100a path with the CPU oracle (needs a B200).

Criteria: residual per cell within 1e-12 of the oracle,
relative to max(|R|, S) with S = sum of |face flux|/VOL of the cell; stage
outputs and fields after many cycles within the tolerances written per test.
"""
import numpy as np
import pytest

from finflo_b200.gpu import GpuSolver
from oracle.oracle import Oracle
from tests.util import hist_close, flux_scale, interior, make_pair

pytestmark = pytest.mark.gpu

RES = ("DRO", "DM", "DN", "DW", "DE")


def _setup(ni=17, nj=9, nk=9, predgs_full=0, **kw):
    bg, bc, prm, fs = make_pair(ni, nj, nk, **kw)
    prm.predgs_full = predgs_full
    o = Oracle(bc, prm)
    o.start()
    g = GpuSolver(0)
    bid = g.add_block(bg, prm)
    g.upload(bid)
    g.start(bid)
    return g, bid, bg, o, bc, prm


def _cmp_state(g, bid, bg, bc, names, rtol):
    d = g.download(bid, names)
    for n in names:
        ref, got = bc.arrays[n], d[n]
        scale = np.abs(ref).max() + 1e-300
        err = np.abs(got - ref).max() / scale
        assert err <= rtol, (n, err)


@pytest.mark.parametrize("dims", [(17, 9, 9), (33, 17, 9)])
def test_statim_boundi(gpu_lib, dims):
    g, bid, bg, o, bc, prm = _setup(*dims)
    g.sync()
    _cmp_state(g, bid, bg, bc, ["RO", "P", "PDIFF", "TEMP", "U", "V", "W", "C", "E", "VIS", "CH",
                                 "DRDP", "DRDH", "RM", "RN", "RW", "EPS2", "VIST"], 1e-14)
    g.close()


@pytest.mark.parametrize("dims,inter", [((17, 9, 9), 3), ((33, 17, 9), 3), ((17, 9, 5), -3), ((17, 9, 9), 55)])
def test_residual(gpu_lib, dims, inter):
    g, bid, bg, o, bc, prm = _setup(*dims, inter=inter)
    o.statim(); o.adjuin(); o.residu(1, 1)
    g.residu(bid, 1, 1)
    g.sync()
    d = g.download(bid, list(RES) + ["S11", "S12", "W12", "DTDX", "DTDZ"])
    S = flux_scale(o, bc)
    for n in RES:
        ref = interior(bc, bc.arrays[n]); got = interior(bg, d[n])
        den = np.maximum(np.abs(ref), S[n]) + 1e-300
        err = (np.abs(got - ref) / den).max()
        assert err <= 1e-12, (n, err)
    # gradients: interior + first ghost layer
    for n in ("S11", "S12", "W12", "DTDX", "DTDZ"):
        ref = bc.arrays[n].reshape(bc.kmax + 4, bc.jmax + 4, bc.imax + 4)[1:-1, 1:-1, 1:-1]
        got = d[n].reshape(bc.kmax + 4, bc.jmax + 4, bc.imax + 4)[1:-1, 1:-1, 1:-1]
        err = np.abs(got - ref).max() / (np.abs(ref).max() + 1e-300)
        assert err <= 1e-12, (n, err)
    g.close()


def test_resl2(gpu_lib):
    g, bid, bg, o, bc, prm = _setup()
    o.statim(); o.adjuin(); o.residu(1, 1)
    g.residu(bid, 1, 1)
    r_g = g.resl2(bid)
    r_c = o.resl2()
    np.testing.assert_allclose(r_g, r_c, rtol=1e-10, atol=1e-300)
    g.close()


@pytest.mark.parametrize("dims", [(17, 9, 9), (25, 13, 7), (17, 65, 65), (9, 41, 19)])
def test_imps_lusgs(gpu_lib, dims):
    """The GPU hyperplane LU-SGS solves the reference's triangular systems
    (incl. the dropped i+1 coupling in the last j row of PREDGS)."""
    g, bid, bg, o, bc, prm = _setup(*dims)
    o.statim(); o.adjuin(); o.residu(1, 1)
    g.residu(bid, 1, 1)
    # same residual on both sides, then IMPS
    g.sync()
    bg_res = g.download(bid, list(RES))
    for n in RES:
        bc.arrays[n][:] = bg_res[n]
    o.imps(1)
    g.imps(bid, 1)
    g.sync()
    d = g.download(bid, list(RES) + ["DTL"])
    for n in list(RES) + ["DTL"]:
        ref = interior(bc, bc.arrays[n]); got = interior(bg, d[n])
        err = np.abs(got - ref).max() / (np.abs(ref).max() + 1e-300)
        assert err <= 1e-11, (n, err)
    g.close()


@pytest.mark.parametrize("kind", ["lines", "hyperplane", "pipe"])
def test_imps_lusgs_predgs_full(gpu_lib, kind, monkeypatch):
    """predgs_full: the lower sweep keeps the row-JMAX i+1 coupling that the
    reference's PREDGS drops (imps4.f:1460); every sweep kernel against the
    oracle."""
    monkeypatch.setenv("FINFLO_LUSGS", kind)
    g, bid, bg, o, bc, prm = _setup(33, 17, 17, predgs_full=1)
    want = {"pipe": 3, "lines": 1, "hyperplane": 2}[kind]
    assert g.lusgs_kind(bid) % 100 == want
    o.statim(); o.adjuin(); o.residu(1, 1)
    g.residu(bid, 1, 1)
    g.sync()
    bg_res = g.download(bid, list(RES))
    for n in RES:
        bc.arrays[n][:] = bg_res[n]
    o.imps(1)
    g.imps(bid, 1)
    g.sync()
    d = g.download(bid, list(RES))
    for n in RES:
        ref = interior(bc, bc.arrays[n]); got = interior(bg, d[n])
        err = np.abs(got - ref).max() / (np.abs(ref).max() + 1e-300)
        assert err <= 1e-11, (n, err)
    g.close()


def test_cycles_predgs_full_match_oracle(gpu_lib):
    """30 graph-captured cycles with predgs_full against the oracle."""
    g, bid, bg, o, bc, prm = _setup(17, 9, 9, predgs_full=1)
    n = 30
    hist = g.cycles(n, bid, icycle0=1, use_graph=True)
    ref = np.array([o.cycle(i + 1)[0] for i in range(n)])
    hist_close(hist[:, :5], ref, 1e-8)
    g.close()


def test_fin(gpu_lib):
    g, bid, bg, o, bc, prm = _setup()
    o.statim(); o.adjuin(); o.residu(1, 1); o.imps(1)
    g.residu(bid, 1, 1)    # same ghost updates (REFCEN, INLET/OUTLET) on both sides
    g.sync()
    for n in RES:
        bg.arrays[n][:] = bc.arrays[n]
    g.upload(bid, list(RES))
    dm_g = g.fin(bid)
    o.fin_limits()
    _cmp_state(g, bid, bg, bc, ["TEMP", "U", "V", "W", "PDIFF", "P"], 1e-15)
    dm_c = np.abs(interior(bc, bc.arrays["DE"])).max()
    assert abs(dm_g - dm_c) <= 1e-15 * dm_c
    g.close()


@pytest.mark.parametrize("use_graph", [False, True])
def test_cycles_match_oracle(gpu_lib, use_graph):
    """30 full cycles: fields and residual history against the oracle."""
    g, bid, bg, o, bc, prm = _setup(17, 9, 9)
    n = 30
    hist = g.cycles(n, bid, icycle0=1, use_graph=use_graph)
    ref = np.array([o.cycle(i + 1)[0] for i in range(n)])
    hist_close(hist[:, :5], ref, 1e-8)
    d = g.download(bid, ["TEMP", "U", "V", "W", "PDIFF"])
    for nme in d:
        a = interior(bg, d[nme]); b = interior(bc, bc.arrays[nme])
        rel = np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-300)
        assert rel <= 1e-10, (nme, rel)
    g.close()


def test_fp32_lusgs_converges_to_fp64_answer(gpu_lib):
    """FP32 implicit operator: the residual stays FP64, so the fixed point is
    the FP64 one; after the same cycles the fields differ by a bounded amount."""
    g, bid, bg, o, bc, prm = _setup(17, 9, 9)
    prm32 = type(prm).from_buffer_copy(prm)
    prm32.lusgs_fp32 = 1
    g2 = GpuSolver(0)
    bg2 = make_pair(17, 9, 9)[0]
    b2 = g2.add_block(bg2, prm32)
    g2.upload(b2)
    g2.start(b2)
    h64 = g.cycles(150, bid)
    h32 = g2.cycles(150, b2)
    assert np.isfinite(h32).all()
    d64 = g.download(bid, ["TEMP", "U", "PDIFF"])
    d32 = g2.download(b2, ["TEMP", "U", "PDIFF"])
    for n in d64:
        a, b = interior(bg, d64[n]), interior(bg2, d32[n])
        rel = np.linalg.norm(a - b) / np.linalg.norm(b)
        assert rel < 1e-3, (n, rel)
    # both runs must be converging
    assert h32[-1, 0] < h32[0, 0] and h64[-1, 0] < h64[0, 0]
    g.close(); g2.close()


@pytest.mark.parametrize("dims", [(33, 33, 33), (17, 65, 65)])
def test_line_and_hyperplane_sweeps_agree(gpu_lib, dims, monkeypatch):
    """The cluster line-wavefront LU-SGS and the cooperative hyperplane kernel
    solve the same triangular systems."""
    g1, b1, bg1, o, bc, prm = _setup(*dims)
    assert g1.lusgs_kind(b1) % 100 == 1
    monkeypatch.setenv("FINFLO_LUSGS", "hyperplane")
    g2 = GpuSolver(0)
    bg2 = make_pair(*dims)[0]
    b2 = g2.add_block(bg2, prm)
    assert g2.lusgs_kind(b2) % 100 == 2
    g2.upload(b2)
    g2.start(b2)
    for g, b in ((g1, b1), (g2, b2)):
        g.residu(b, 1, 1)
        g.imps(b, 1)
    d1 = g1.download(b1, list(RES))
    d2 = g2.download(b2, list(RES))
    for n in RES:
        a, c = interior(bg1, d1[n]), interior(bg2, d2[n])
        err = np.abs(a - c).max() / (np.abs(c).max() + 1e-300)
        assert err <= 1e-12, (n, err)
    g1.close(); g2.close()


@pytest.mark.parametrize("dims", [(33, 33, 33), (17, 65, 65), (21, 40, 22)])
def test_pipe_and_hyperplane_sweeps_agree(gpu_lib, dims, monkeypatch):
    """The pipelined tile-wavefront LU-SGS (tiles synchronised point to point
    by mbarriers, edge products pushed through DSMEM) solves the same
    triangular systems as the cooperative hyperplane kernel, including
    partial tiles (j and k line counts that are not multiples of the tile)."""
    monkeypatch.setenv("FINFLO_LUSGS", "pipe")
    g1, b1, bg1, o, bc, prm = _setup(*dims)
    assert g1.lusgs_kind(b1) % 100 == 3
    monkeypatch.setenv("FINFLO_LUSGS", "hyperplane")
    g2 = GpuSolver(0)
    bg2 = make_pair(*dims)[0]
    b2 = g2.add_block(bg2, prm)
    assert g2.lusgs_kind(b2) % 100 == 2
    g2.upload(b2)
    g2.start(b2)
    for g, b in ((g1, b1), (g2, b2)):
        g.residu(b, 1, 1)
        g.imps(b, 1)
    d1 = g1.download(b1, list(RES))
    d2 = g2.download(b2, list(RES))
    for n in RES:
        a, c = interior(bg1, d1[n]), interior(bg2, d2[n])
        err = np.abs(a - c).max() / (np.abs(c).max() + 1e-300)
        assert err <= 1e-12, (n, err)
    g1.close(); g2.close()


def test_pipe_cycles_match_oracle(gpu_lib, monkeypatch):
    """Graph-captured cycles with the pipelined sweep against the oracle."""
    monkeypatch.setenv("FINFLO_LUSGS", "pipe")
    g, bid, bg, o, bc, prm = _setup(33, 17, 17)
    assert g.lusgs_kind(bid) % 100 == 3
    n = 20
    hist = g.cycles(n, bid, icycle0=1, use_graph=True)
    ref = np.array([o.cycle(i + 1)[0] for i in range(n)])
    hist_close(hist[:, :5], ref, 1e-9)
    g.close()


@pytest.mark.parametrize("nlev,dims", [(2, (17, 9, 9)), (3, (33, 17, 17))])
def test_multigrid_cycles_match_oracle(gpu_lib, nlev, dims):
    """FAS V-cycles (TRANSF, FORCFU, ADDRES, INTERP, coarse FLUXDO/first-order
    Roe, coarse LU-SGS) against the oracle: residual history and fields."""
    from finflo_b200 import case
    from oracle.oracle import OracleMG
    lv_g, prms, fs = case.bump_case_mg(*dims, nlev=nlev)
    lv_c, _, _ = case.bump_case_mg(*dims, nlev=nlev)
    om = OracleMG(lv_c, prms)
    om.start()
    g = GpuSolver(0)
    bid = g.add_levels(lv_g, prms)
    for b in range(len(lv_g)):
        g.upload(bid + b)
    g.start(bid)
    n = 12
    hist = g.cycles(n, bid, icycle0=1, use_graph=True)
    ref = np.array([om.cycle(i + 1)[0] for i in range(n)])
    hist_close(hist[:, :5], ref, 1e-7)
    d = g.download(bid, ["TEMP", "U", "V", "PDIFF"])
    for nme in d:
        a = interior(lv_g[0], d[nme]); b = interior(lv_c[0], lv_c[0].arrays[nme])
        rel = np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-300)
        assert rel <= 1e-9, (nme, rel)
    g.close()


@pytest.mark.parametrize("kind", ["lockstep", "lines", "hyperplane"])
def test_multiblock_cycles_match_oracle(gpu_lib, kind, monkeypatch):
    """Periodic box of 2x2x2 uneven blocks: all-block BOUNDI with device
    CONNEC, against the oracle's multi-block cycle.  lockstep: each stage
    over all blocks with both LU-SGS sweeps of all blocks in one batched
    launch; lines / hyperplane: concurrent per-block chains in one captured
    graph, with that sweep kernel."""
    from finflo_b200 import case
    from oracle.oracle import OracleMB
    if kind == "lockstep":
        monkeypatch.setenv("FINFLO_MB_LOCKSTEP", "1")
    if kind == "hyperplane":
        monkeypatch.setenv("FINFLO_LUSGS", "hyperplane")
    sizes = ([9, 13], [7, 11], [9, 6])
    bg, pg, _ = case.periodic_box_case(nb=(2, 2, 2), sizes=sizes)
    bc, pc, _ = case.periodic_box_case(nb=(2, 2, 2), sizes=sizes)
    om = OracleMB(bc, pc)
    om.start()
    g = GpuSolver(0)
    for b, p in zip(bg, pg):
        bid = g.add_block(b, p)
        g.upload(bid)
    g.start_all()
    n = 15
    hist = g.cycles_all(n, icycle0=1, use_graph=True)
    ref = np.array([om.cycle(i + 1)[0] for i in range(n)])
    hist_close(hist[:, :5], ref, 1e-9)
    for bid in range(len(bg)):
        d = g.download(bid, ["TEMP", "U", "V", "W", "PDIFF"])
        for nme in d:
            a = interior(bg[bid], d[nme]); b = interior(bc[bid], bc[bid].arrays[nme])
            # PDIFF = p - p_inf starts at zero in the box: scale it by p_inf
            scale = np.linalg.norm(b) if nme != "PDIFF" else pc[bid].frspre * np.sqrt(b.size)
            rel = np.linalg.norm(a - b) / (scale + 1e-300)
            assert rel <= 1e-11, (bid, nme, rel)
    g.close()


@pytest.mark.parametrize("turb", [None, "sst"])
@pytest.mark.parametrize("mode", ["lockstep", "branches"])
def test_multiblock_multigrid_matches_oracle(gpu_lib, turb, mode, monkeypatch):
    """Eight uneven blocks of the spanwise-varying bump (1:1 cuts, periodic
    z), two multigrid levels each, BOUNDI/CONNEC over the level-1 blocks,
    against the oracle's multi-block multigrid cycle: stage by stage over
    all blocks with each level's sweeps batched (lockstep), or per-block
    V-cycles as concurrent graph branches."""
    from finflo_b200 import case
    from oracle.oracle import OracleMBMG
    if mode == "lockstep":
        monkeypatch.setenv("FINFLO_MB_LOCKSTEP", "1")
    kw = dict(cells=(40, 16, 16), nb=(2, 2, 2), nlev=2, h1=1e-3, reynolds=1e4, mach=0.5, cfl=2.0, cfll=2.0,
              lusgs_fp32=False, coarse_fp32=False, turbulence=turb)
    if turb == "sst":
        kw.update(reynolds=1e6, mach=0.6, h1=1e-4, cfl=1.0, cfll=1.0)
    bg, pg, _ = case.bump_multiblock_case(**kw)
    bc, pc, _ = case.bump_multiblock_case(**kw)
    om = OracleMBMG(bc, pc)
    om.start()
    g = GpuSolver(0)
    ids = g.add_multiblock(bg, pg)
    for bid in range(len(g.blocks)):
        g.upload(bid)
    g.start_all()
    n = 10
    hist = g.cycles_all(n, icycle0=1, use_graph=True)
    ref = np.array([om.cycle(i + 1)[0] for i in range(n)])
    hist_close(hist[:, :5], ref, 1e-8 if turb else 1e-9)
    names = ["TEMP", "U", "V", "W", "PDIFF"] + (["RK", "REPS"] if turb else [])
    for k, bid in enumerate(ids):
        d = g.download(bid, names)
        for nme in names:
            a = interior(bg[k][0], d[nme]); b = interior(bc[k][0], bc[k][0].arrays[nme])
            scale = np.linalg.norm(b) if nme != "PDIFF" else pc[k][0].frspre * np.sqrt(b.size)
            rel = np.linalg.norm(a - b) / (scale + 1e-300)
            assert rel <= 1e-9, (k, nme, rel)
    g.close()


def test_halo_loopback_matches_oracle(gpu_lib):
    """Every 1:1 patch treated as remote: the device halo pack / unpack
    through one buffer (what a send/recv between GPUs moves) and the phased
    cycle reproduce the oracle's multi-block cycles."""
    import torch
    from finflo_b200 import case
    from finflo_b200 import dist as fd
    from finflo_b200.case import Block
    from oracle.oracle import OracleMB
    sizes = ([9, 12], [7, 10], [8])
    bg, pg, _ = case.periodic_box_case(nb=(2, 2, 1), sizes=sizes)
    bc, pc, _ = case.periodic_box_case(nb=(2, 2, 1), sizes=sizes)
    om = OracleMB(bc, pc)
    om.start()
    items, off = [], 0
    for l in fd.links(bg):
        items.append(fd.HaloPlan._item(l.src, 0, off, l.pa))
        items.append(fd.HaloPlan._item(l.dst, 1, off, l.pa))
        off += l.doubles
    g = GpuSolver(0)
    for b, p in zip(bg, pg):
        pats = [fd._copy_patch(pa) for pa in b.patches]
        for pa in pats:
            pa.ibtype = -1 - pa.ibtype
        bid = g.add_block(Block(b.imax, b.jmax, b.kmax, b.arrays, pats, b.nodes), p)
        g.upload(bid)
    buf = torch.zeros(off, dtype=torch.float64, device="cuda:0")
    torch.cuda.synchronize()
    g.halo_plan(items, buf.data_ptr(), buf.data_ptr())
    g.mb_phase(fd.PHASE_BOUNDI_A, 1, False)
    g.mb_phase(fd.PHASE_B, 1, False)
    g.sync()
    for bid in range(len(bg)):
        g._old_copies(bid)
    n = 12
    g.reserve_history(n)
    for i in range(n):
        g.mb_phase(fd.PHASE_CYCLE_A, i + 1, True)
        g.mb_phase(fd.PHASE_B, i + 1, True)
        g.mb_phase(fd.PHASE_RECORD, i + 1, True)
    hist = g.history(n)
    ref = np.array([om.cycle(i + 1)[0] for i in range(n)])
    hist_close(hist[:, :5], ref, 1e-9)
    for bid in range(len(bg)):
        d = g.download(bid, ["TEMP", "U", "V", "W", "PDIFF"])
        for nme in d:
            a = interior(bg[bid], d[nme]); b = interior(bc[bid], bc[bid].arrays[nme])
            # PDIFF = p - p_inf starts at zero in the box: scale it by p_inf
            scale = np.linalg.norm(b) if nme != "PDIFF" else pc[bid].frspre * np.sqrt(b.size)
            rel = np.linalg.norm(a - b) / (scale + 1e-300)
            assert rel <= 1e-11, (bid, nme, rel)
    g.close()
