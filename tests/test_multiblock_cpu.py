"""Multi-block oracle (CONNEC, all-block BOUNDI and cycles) on the CPU."""
import numpy as np
import pytest

from finflo_b200 import case
from oracle.oracle import OracleMB

RES = ("DRO", "DM", "DN", "DW", "DE")


def _residuals(blocks, prms):
    om = OracleMB(blocks, prms)
    om.boundi()
    for o in om.blocks:
        o.statim(); o.adjuin(); o.residu(1, 1)
    return om


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_split_block_residual_is_bitwise_the_unsplit_one(axis):
    """A periodic box cut in two along one axis and joined by 1:1 patches has
    exactly the residual of the uncut box (periodic onto itself)."""
    full = [[16], [6], [5]]
    full[axis] = [7 + 2 * axis, 9]
    cut = [list(v) for v in full]
    one = [[sum(v)] for v in full]
    bl, pr, _ = case.periodic_box_case(nb=tuple(len(v) for v in cut), sizes=cut)
    bs, ps, _ = case.periodic_box_case(nb=(1, 1, 1), sizes=one)
    _residuals(bl, pr); _residuals(bs, ps)
    ax = 2 - axis    # interior() is (k, j, i)
    for n in RES:
        a = np.concatenate([b.interior(n) for b in bl], axis=ax)
        assert np.array_equal(a, bs[0].interior(n)), n


def test_periodic_box_conserves_and_preserves_free_stream():
    bl, pr, _ = case.periodic_box_case(nb=(2, 2, 2), sizes=([5, 7], [6, 4], [5, 3]))
    _residuals(bl, pr)
    scale = max(np.abs(b.interior("DE")).max() for b in bl)
    for n in RES:
        tot = sum((b.interior(n) * b.interior("VOL")).sum() for b in bl)
        assert abs(tot) <= 1e-13 * scale, (n, tot)
    bl, pr, _ = case.periodic_box_case(nb=(2, 2, 1), sizes=([5, 7], [6, 4], [5]), amp=0.0)
    _residuals(bl, pr)
    for b in bl:
        for n in RES:
            assert np.abs(b.interior(n)).max() <= 1e-9, n


def test_box_block_sizes_are_seeded_and_in_range():
    s = case.box_block_sizes()
    assert s == case.box_block_sizes()
    assert all(16 <= v <= 96 and v % 4 == 0 for d in s for v in d)
    assert [len(d) for d in s] == [4, 3, 2]
    cells = sum(a * b * c for a in s[0] for b in s[1] for c in s[2])
    assert 5.4e6 <= cells <= 6.6e6


def test_multiblock_cycles_converge():
    """Local time steps drive the periodic entropy wave to the uniform steady
    state: the density residual falls steadily over 40 cycles."""
    bl, pr, fs = case.periodic_box_case(nb=(2, 1, 1), sizes=([6, 8], [6], [4]))
    om = OracleMB(bl, pr)
    om.start()
    hist = np.array([om.cycle(i + 1)[0] for i in range(40)])
    assert np.isfinite(hist).all()
    r = np.sqrt(hist[:, 0])
    assert (np.diff(r) < 0).all() and r[-1] < 0.5 * r[0]


def _mbmg_case(turbulence=None, cells=(40, 16, 16), nb=(2, 2, 2), nlev=2):
    from finflo_b200 import case
    kw = dict(h1=1e-3, reynolds=1e4, mach=0.5, cfl=2.0, cfll=2.0, lusgs_fp32=False, coarse_fp32=False,
              turbulence=turbulence)
    if turbulence == "sst":
        kw.update(reynolds=1e6, mach=0.6, h1=1e-4, cfl=1.0, cfll=1.0)
    return case.bump_multiblock_case(cells=cells, nb=nb, nlev=nlev, **kw)


def test_multiblock_multigrid_one_block_equals_the_block_cycle():
    """With one block (no 1:1 patches) the multi-block multigrid cycle is the
    single-block V-cycle: identical history and fields, laminar and SST."""
    from finflo_b200 import case
    from oracle.oracle import OracleMG, OracleMBMG
    for turb in (None, "sst"):
        kw = dict(turbulence=turb, reynolds=1e6 if turb else 1e4, h1=1e-4 if turb else 1e-3)
        l1, p1, _ = case.bump_case_mg(17, 9, 9, nlev=2, **kw)
        l2, p2, _ = case.bump_case_mg(17, 9, 9, nlev=2, **kw)
        a, b = OracleMG(l1, p1), OracleMBMG([l2], [p2])
        a.start()
        b.start()
        for ic in range(1, 4):
            ra, da = a.cycle(ic)
            rb, db = b.cycle(ic)
            np.testing.assert_array_equal(ra, rb)
            assert da == db
        for n in ("TEMP", "U", "PDIFF", "RK"):
            np.testing.assert_array_equal(l1[0].arrays[n], l2[0].arrays[n])


def test_multiblock_multigrid_converges():
    """Eight uneven blocks of the spanwise-varying bump with two multigrid
    levels each: the oracle's multi-block multigrid cycles run and the
    density residual falls."""
    from oracle.oracle import OracleMBMG
    bl, bp, _ = _mbmg_case()
    om = OracleMBMG(bl, bp)
    om.start()
    h = [om.cycle(i + 1)[0][0] for i in range(30)]
    assert np.all(np.isfinite(h))
    assert min(h[-5:]) < 0.3 * h[0]
