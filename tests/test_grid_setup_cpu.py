"""The host set-up (finflo_b200/grid.py, case.py) against the oracle's
restatement of the reference's (oracle/finflo_oracle_grid.c):

* GRIDEX ghost nodes + AREVC1 faces, normals, volumes, centres and D1D2D3
  (gluebm.f:1029, 1586, 2326) of the interior cells and the first ghost
  layer, edges and corners included;
* LUMPA1 / LUMPVS coarse faces, volumes and centres (gluebm.f:2194, 2256)
  of the interior of two coarse levels;
* PICK_XYZ wall points and WALL_DIST / LUMP_DIST wall distance
  (gluebm.f:9452, 9533, 9562),

all equal to the bit, on a bump channel with a spanwise-varying bump
(warped faces) and on a box with every interior node moved."""
import ctypes

import numpy as np
import pytest

from finflo_b200 import case, grid
from finflo_b200.case import SLOTS
from oracle.oracle import OrcBlock, lib

NAMES = list(grid.METRIC_NAMES)


def _orc(imax, jmax, kmax, patches=()):
    nt = grid.strides(imax, jmax, kmax)[2]
    arrays = {n: np.zeros(nt) for n in SLOTS}
    pa = (case.FFPatch * max(1, len(patches)))(*patches)
    ob = OrcBlock()
    ob.imax, ob.jmax, ob.kmax, ob.npatch = imax, jmax, kmax, len(patches)
    ob.patch = ctypes.cast(pa, ctypes.POINTER(case.FFPatch))
    for i, n in enumerate(SLOTS):
        ob.a[i] = arrays[n].ctypes.data
    return ob, arrays, pa


def _nodes(kind):
    if kind == "bump":
        return grid.bump_nodes(33, 17, 17, h1=1e-3, amp=0.1, span_amp=0.5, zlen=1.0)
    X, Y, Z = grid.box_nodes(np.linspace(0, 1, 21), np.linspace(0, 0.5, 13), np.linspace(0, 0.3, 9))
    rng = np.random.default_rng(3)
    for A in (X, Y, Z):
        A[1:-1, 1:-1, 1:-1] += 0.015 * rng.uniform(-1, 1, A[1:-1, 1:-1, 1:-1].shape)
    return X, Y, Z


def _ref_metrics(X, Y, Z):
    imax, jmax, kmax = X.shape[2] - 1, X.shape[1] - 1, X.shape[0] - 1
    ob, arrays, keep = _orc(imax, jmax, kmax)
    c = [np.ascontiguousarray(a) for a in (X, Y, Z)]
    lib().orc_grid_metrics(ctypes.byref(ob), *(a.ctypes.data_as(ctypes.c_void_p) for a in c))
    return ob, arrays, keep


@pytest.mark.parametrize("kind", ["bump", "warped"])
def test_fine_metrics_equal_the_reference_construction(kind):
    X, Y, Z = _nodes(kind)
    _, ref, _ = _ref_metrics(X, Y, Z)
    m = grid.compute_metrics(X, Y, Z)
    sh = (m.kmax + 4, m.jmax + 4, m.imax + 4)
    for n in NAMES:   # cells 0..MAX+1: the interior and the first ghost layer
        a = m.arrays[n].reshape(sh)[1:-1, 1:-1, 1:-1]
        r = ref[n].reshape(sh)[1:-1, 1:-1, 1:-1]
        np.testing.assert_array_equal(a, r, err_msg=n)


@pytest.mark.parametrize("kind", ["bump", "warped"])
def test_coarse_metrics_equal_the_reference_lumping(kind):
    X, Y, Z = _nodes(kind)
    ob, _, keep = _ref_metrics(X, Y, Z)
    levels = grid.mg_metrics(X, Y, Z, 3)
    prev = ob
    held = [keep]
    for lev in (1, 2):
        m = levels[lev]
        obc, ref, kc = _orc(m.imax, m.jmax, m.kmax)
        held.append(kc)
        lib().orc_grid_lump(ctypes.byref(prev), ctypes.byref(obc))
        sh = (m.kmax + 4, m.jmax + 4, m.imax + 4)
        for n in NAMES:
            sl = [slice(2, m.kmax + 2), slice(2, m.jmax + 2), slice(2, m.imax + 2)]
            if n[0] == "A" and n[1] in "123":   # the interior faces, the last one included
                d = int(n[1]) - 1
                sl[2 - d] = slice(2, (m.imax, m.jmax, m.kmax)[d] + 3)
            np.testing.assert_array_equal(m.arrays[n].reshape(sh)[tuple(sl)], ref[n].reshape(sh)[tuple(sl)],
                                          err_msg=f"level {lev + 1} {n}")
        prev = obc


def test_wall_distance_equals_the_reference_search():
    levels, prms, fs = case.bump_case_mg(33, 17, 17, nlev=3, turbulence="sst", reynolds=1e6, h1=1e-4,
                                         span_amp=0.5, zlen=1.0)
    f = levels[0]
    ob, ref, keep = _orc(f.imax, f.jmax, f.kmax, f.patches)
    for n in NAMES:
        ref[n][:] = f.arrays[n]
    L = lib()
    ptr = (ctypes.POINTER(OrcBlock) * 1)(ctypes.pointer(ob))
    npts = L.orc_wall_points(ptr, 1, None)
    pts = np.zeros(3 * npts)
    L.orc_wall_points(ptr, 1, pts.ctypes.data_as(ctypes.c_void_p))
    pts = pts.reshape(-1, 3)
    np.testing.assert_array_equal(case.wall_points(f.nodes, f.patches), pts)
    L.orc_wall_distance(ctypes.byref(ob), pts.ctypes.data_as(ctypes.c_void_p), npts)
    np.testing.assert_array_equal(f.arrays["DISTW"], ref["DISTW"])
    # the coarse levels' interior: the mean of the children (LUMP_DIST)
    prev, hold = ob, [keep]
    for lev in (1, 2):
        c = levels[lev]
        obc, rc, kc = _orc(c.imax, c.jmax, c.kmax)
        hold.append(kc)
        for n in NAMES:
            rc[n][:] = c.arrays[n]
        L.orc_grid_lump(ctypes.byref(prev), ctypes.byref(obc))
        np.testing.assert_array_equal(c.interior("DISTW"),
                                      rc["DISTW"].reshape(c.kmax + 4, c.jmax + 4, c.imax + 4)[2:-2, 2:-2, 2:-2])
        prev = obc
