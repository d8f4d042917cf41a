"""1:1 patches in every orientation (ICON(14), gluebm.f:8188).

Two blocks of a Cartesian box meet at an interface; the second block's
index axes are turned by each of the 24 proper rotations of the index cube,
so the interface lies on any of its six faces in any of the four turns.
ORIENT (gluebm.f:8506, restated as case.orient) finds ICON(14) from the
patch corners (CORNER gluebm.f:2480), and the oracle's CONNEC, with the
export / import orders and PERMUT's turn (gluebm.f:5096, 5174, 4868), must
fill each block's ghost cells with the neighbour's cells at the same place:
a linear field of the cell centres arrives exactly where it belongs.
"""
import ctypes
import itertools

import numpy as np
import pytest

from finflo_b200 import case, grid
from oracle.oracle import Oracle

H = (0.13, 0.21, 0.34)            # cell sizes in x, y, z (distinct: a transposition shows)
CELLS_A, CELLS_B = (4, 5, 3), (3, 5, 3)   # block A cells, block B cells (before its turn)


def rotations():
    """The 24 index-axis rotations (perm, flips) with determinant +1: new
    axis n is old axis perm[n], reversed where flips[n]."""
    out = []
    for perm in itertools.permutations(range(3)):
        for flips in itertools.product((False, True), repeat=3):
            m = np.zeros((3, 3))
            for n, o in enumerate(perm):
                m[n, o] = -1.0 if flips[n] else 1.0
            if round(np.linalg.det(m)) == 1:
                out.append((perm, flips))
    return out


def _turn(a, perm, flips):
    """A node array [k, j, i] re-indexed by the rotation."""
    t = a.transpose(2, 1, 0).transpose(perm)        # [i', j', k'] from [i, j, k]
    for n in range(3):
        if flips[n]:
            t = np.flip(t, axis=n)
    return np.ascontiguousarray(t.transpose(2, 1, 0))


def _new_face(iface, perm, flips):
    """The face of the turned block that was face iface."""
    d, hi = (iface - 1) % 3, iface > 3
    n = perm.index(d)
    hi = hi != flips[n]
    return n + 1 + (3 if hi else 0)


def _full_ranges(iface, dims):
    d = (iface - 1) % 3
    t = [x for q, x in enumerate(dims) if q != d]
    return (1, t[0]), (1, t[1])


def _pair(perm, flips):
    na, nb = CELLS_A, CELLS_B
    xa = np.arange(na[0] + 1) * H[0]
    xb = (na[0] + np.arange(nb[0] + 1)) * H[0]
    y = np.arange(na[1] + 1) * H[1]
    z = np.arange(na[2] + 1) * H[2]
    XA, YA, ZA = grid.box_nodes(xa, y, z)
    XB, YB, ZB = (_turn(a, perm, flips) for a in grid.box_nodes(xb, y, z))
    dims_b = tuple(nb[perm[n]] for n in range(3))
    fb = _new_face(1, perm, flips)                   # block B's old i-low face
    pa = case._patch(grid.BC_CON, 4, *_full_ranges(4, na), ibtype=1)
    pb = case._patch(grid.BC_CON, fb, *_full_ranges(fb, dims_b), ibtype=0)
    pa.nface, pb.nface = fb, 4
    pa.n1a = pa.n2a = pb.n1a = pb.n2a = 1
    A = case.new_block(XA, YA, ZA, [pa])
    B = case.new_block(XB, YB, ZB, [pb])
    assert (B.imax, B.jmax, B.kmax) == dims_b
    case.orient_connections([A, B])
    return A, B


def _field(blk):
    return 1.0 + 0.3 * blk.arrays["XC"] + 0.7 * blk.arrays["YC"] + 1.3 * blk.arrays["ZC"]


def _ghosts(blk, pa):
    """Flat indices of the two ghost layers behind the patch."""
    d = (pa.iface - 1) % 3
    out = []
    for g in (1, 2):
        layer = 1 - g if pa.iface <= 3 else (blk.imax, blk.jmax, blk.kmax)[d] + g
        for c in range(pa.r2a, pa.r2b + 1):
            for a in range(pa.r1a, pa.r1b + 1):
                i, j, k = (layer, a, c) if d == 0 else ((a, layer, c) if d == 1 else (a, c, layer))
                out.append(((k + 1) * (blk.jmax + 4) + (j + 1)) * (blk.imax + 4) + (i + 1))
    return np.array(out)


@pytest.mark.parametrize("rot", range(24))
def test_connection_fills_the_ghosts_with_the_neighbour_cells(rot):
    perm, flips = rotations()[rot]
    A, B = _pair(perm, flips)
    fc = case.FlowConditions()
    prm = case.make_params(fc, A.dims)
    oa, ob = Oracle(A, prm), Oracle(B, prm)
    for blk in (A, B):
        blk.arrays["TEMP"][:] = _field(blk)
        blk.arrays["TEMP"][_ghosts(blk, blk.patches[0])] = -1.0
    L = oa.L
    L.orc_connec_patch(ctypes.byref(oa.ob), ctypes.byref(A.patches[0]), ctypes.byref(ob.ob))
    L.orc_connec_patch(ctypes.byref(ob.ob), ctypes.byref(B.patches[0]), ctypes.byref(oa.ob))
    for blk in (A, B):
        g = _ghosts(blk, blk.patches[0])
        np.testing.assert_allclose(blk.arrays["TEMP"][g], _field(blk)[g], rtol=0, atol=1e-12)


def test_rotations_cover_every_face_and_turn():
    seen = set()
    for perm, flips in rotations():
        A, B = _pair(perm, flips)
        seen.add((B.patches[0].iface, A.patches[0].iori))
        assert A.patches[0].iori >= 0 and B.patches[0].iori >= 0
    assert {f for f, _ in seen} == set(range(1, 7))
    assert {t for _, t in seen} == {0, 1, 2, 3}


def test_cut_and_periodic_patches_of_the_workloads_are_turn_zero():
    it = case.bump_multiblock_blocks(cells=(32, 16, 8), nb=(2, 2, 2), nlev=1, turbulence=None)
    next(it)
    blocks = [lv[0] for lv, _ in it]
    case.orient_connections(blocks)
    assert all(pa.iori == 0 for b in blocks for pa in b.patches if pa.ityp == grid.BC_CON)
    bx, _, _ = case.periodic_box_case(nb=(2, 2, 2), sizes=([5, 6], [4, 5], [3, 4]))
    case.orient_connections(bx)
    assert all(pa.iori == 0 for b in bx for pa in b.patches)


@pytest.mark.parametrize("rot", [5, 11, 17])
def test_halo_pack_and_unpack_equal_the_connection(rot):
    """The remote form (orc_halo_pack on the donor, orc_halo_unpack on the
    receiver: what crosses between GPUs) of a turned connection fills the
    same ghosts as orc_connec_patch."""
    perm, flips = rotations()[rot]
    A, B = _pair(perm, flips)
    A2, B2 = _pair(perm, flips)
    prm = case.make_params(case.FlowConditions(), A.dims)
    for blk in (A, B, A2, B2):
        blk.arrays["TEMP"][:] = _field(blk)
        blk.arrays["TEMP"][_ghosts(blk, blk.patches[0])] = -1.0
    oa, ob, oa2, ob2 = (Oracle(b, prm) for b in (A, B, A2, B2))
    L = oa.L
    L.orc_connec_patch(ctypes.byref(oa.ob), ctypes.byref(A.patches[0]), ctypes.byref(ob.ob))
    pa = A2.patches[0]
    n = (pa.r1b - pa.r1a + 1) * (pa.r2b - pa.r2a + 1)
    buf = np.zeros(2 * 12 * n)
    L.orc_halo_pack(ctypes.byref(ob2.ob), ctypes.byref(pa), buf.ctypes.data_as(ctypes.c_void_p))
    L.orc_halo_unpack(ctypes.byref(oa2.ob), ctypes.byref(pa), buf.ctypes.data_as(ctypes.c_void_p))
    np.testing.assert_array_equal(A2.arrays["TEMP"], A.arrays["TEMP"])
