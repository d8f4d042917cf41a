"""CPU tests: the oracle's analytic invariants, golden regression vectors and
the C-ABI library's exported symbols (no GPU needed)."""
import ctypes
import math
import os
import re

import numpy as np
import pytest

from finflo_b200 import case, grid
from oracle.oracle import Oracle, roe_face
from tests.util import interior

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _prm():
    fc = case.FlowConditions()
    return case.make_params(fc, (8, 8, 8)), fc.freestream()


def _euler_flux(q, n, gamma):
    ro, u, v, w, p = q
    un = u * n[0] + v * n[1] + w * n[2]
    e = p / (gamma - 1) + 0.5 * ro * (u * u + v * v + w * w)
    return np.array([ro * un, ro * u * un + p * n[0], ro * v * un + p * n[1], ro * w * un + p * n[2],
                     (e + p) * un])


def _cell(q, prm):
    ro, u, v, w, p = q
    t = p / (ro * prm.rgas)
    drdp = 1.0 / (t * prm.rgas)
    e = t * prm.rgas / (prm.gamma - 1)
    drdh = -ro / e / prm.gamma
    c = math.sqrt(max(1.0 / (drdh / ro + drdp), 1.0))
    return [c, drdp, drdh, ro, p]


@pytest.mark.parametrize("intem", [3, -3, 55])
def test_roe_consistency(intem):
    """F(U, U) equals the physical Euler flux (FLUXKE consistency)."""
    prm, fs = _prm()
    q = [fs["rho"] * 1.1, 120.0, -30.0, 15.0, fs["p"] * 0.9]
    n = np.array([0.3, 0.5, 0.81])
    n /= np.linalg.norm(n)
    cl = _cell(q, prm)
    f = roe_face(q, q, q, q, n, 2.0, intem, prm, cl, cl)
    ref = 2.0 * _euler_flux(q, n, prm.gamma)
    np.testing.assert_allclose(f, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


def test_roe_rotational_invariance():
    """Rotating states and face normal together rotates the momentum flux."""
    prm, fs = _prm()
    rng = np.random.default_rng(5)
    ql = [fs["rho"], 150.0, 20.0, -10.0, fs["p"]]
    qr = [fs["rho"] * 1.05, 140.0, 25.0, -5.0, fs["p"] * 1.03]
    n = np.array([0.6, 0.64, 0.48])
    A = np.linalg.qr(rng.standard_normal((3, 3)))[0]
    if np.linalg.det(A) < 0:
        A[:, 0] *= -1

    def rot(q):
        u = A @ np.array(q[1:4])
        return [q[0], *u, q[4]]

    f1 = roe_face(qr, ql, qr, ql, n, 1.0, 3, prm, _cell(qr, prm), _cell(ql, prm))
    f2 = roe_face(rot(qr), rot(ql), rot(qr), rot(ql), A @ n, 1.0, 3, prm, _cell(qr, prm), _cell(ql, prm))
    assert abs(f1[0] - f2[0]) <= 1e-12 * abs(f1[0])
    assert abs(f1[4] - f2[4]) <= 1e-12 * abs(f1[4])
    np.testing.assert_allclose(A @ f1[1:4], f2[1:4], rtol=1e-10, atol=1e-12 * np.abs(f1[1:4]).max())


def _wavy_box(n=9):
    x = np.linspace(0, 1, n)
    X, Y, Z = grid.box_nodes(x, x, x)
    s = 0.03 * np.sin(2 * np.pi * X) * np.sin(2 * np.pi * Y) * np.sin(2 * np.pi * Z)
    return X + s, Y - s, Z + 0.5 * s


def test_metrics_closed_cells():
    X, Y, Z = _wavy_box()
    m = grid.compute_metrics(X, Y, Z)
    a = m.arrays
    im, jm, km = m.imax, m.jmax, m.kmax
    istr, il = im + 4, (im + 4) * (jm + 4)
    for K in range(1, km + 1):
        for J in range(1, jm + 1):
            for I in range(1, im + 1):
                n = grid.sidx(I, J, K, im, jm)
                s = np.zeros(3)
                for dname, st in (("A1", 1), ("A2", istr), ("A3", il)):
                    for lo, sg in ((n, -1), (n + st, 1)):
                        s += sg * a[dname][lo] * np.array([a[dname + "XA"][lo], a[dname + "YA"][lo], a[dname + "ZA"][lo]])
                assert np.abs(s).max() < 1e-13
    assert (interior(m, a["VOL"]) > 0).all() if hasattr(m, "kmax") else True


@pytest.mark.parametrize("flux", list(case.FLUX))
def test_freestream_preservation(flux):
    """Uniform flow on a curved, closed grid: the residual vanishes for every
    IFLUX scheme (the split or averaged fluxes of a uniform state add up to
    the exact flux, up to a constant pressure that a closed cell cancels)."""
    X, Y, Z = _wavy_box()
    fc = case.FlowConditions(mach=0.5, reynolds=1e4)
    fs = fc.freestream()
    im = X.shape[2] - 1
    inl = dict(bounr=fs["rho"], bounu=fs["u"], bounv=0.0, bounw=0.0, bount=fs["t"], bounp=fs["p"], bounpd=0.0)
    pats = [case._patch(grid.BC_INL, 1, (1, im), (1, im), ibtype=4, **inl),
            case._patch(grid.BC_OUT, 4, (1, im), (1, im), ibtype=3, **inl)]
    # flat y and z boundaries: the free stream is tangent there
    for f in (2, 5, 3, 6):
        pats.append(case._patch(grid.BC_MIR, f, (1, im), (1, im)))
    blk = case.new_block(X, Y, Z, pats)
    case.init_freestream(blk, fs, noise=0.0)
    prm = case.make_params(fc, blk.dims)
    prm.flux = case.FLUX[flux]
    o = Oracle(blk, prm)
    o.start()
    o.statim(); o.adjuin(); o.residu(1, 2)
    scale = fs["rho"] * fs["u"] ** 2 * 1.0
    for n in ("DRO", "DM", "DN", "DW", "DE"):
        r = interior(blk, blk.arrays[n]) * interior(blk, blk.arrays["VOL"])
        ref = {"DRO": fs["rho"] * fs["u"], "DE": fs["p"] * fs["u"] * 3.5}.get(n, scale)
        assert np.abs(r).max() < 1e-11 * ref * (1.0 / im) ** 2, n


def test_conservation_telescopes():
    """Sum of VOL*R over the block equals the net boundary flux (interior
    faces cancel in SWEEP)."""
    blk, prm, fs = case.bump_case(13, 7, 5)
    o = Oracle(blk, prm)
    o.start()
    o.statim(); o.adjuin(); o.residu(1, 1)
    tot = sum(np.sum(interior(blk, blk.arrays[n]) * interior(blk, blk.arrays["VOL"])) for n in ["DRO"])
    # boundary flux of mass from the face arrays
    L = o.L
    net = 0.0
    istr, il = blk.imax + 4, (blk.imax + 4) * (blk.jmax + 4)
    for d, st, nmax in ((1, 1, blk.imax), (2, istr, blk.jmax), (3, il, blk.kmax)):
        L.orc_flux_dir(o._b(), o._p(), d, 1)
        F = blk.arrays["F1R"]
        for K in range(1, blk.kmax + 1):
            for J in range(1, blk.jmax + 1):
                for I in range(1, blk.imax + 1):
                    idx = (I, J, K)[d - 1]
                    n = grid.sidx(I, J, K, blk.imax, blk.jmax)
                    if idx == 1:
                        net += F[n]
                    if idx == nmax:
                        net -= F[n + st]
    assert abs(tot - net) <= 1e-12 * (abs(net) + np.abs(blk.arrays["F1R"]).max())


def test_oracle_cycles_converge():
    blk, prm, fs = case.bump_case(17, 9, 9)
    o = Oracle(blk, prm)
    o.start()
    r = [o.cycle(i + 1)[0][0] for i in range(60)]
    assert np.isfinite(r).all()
    assert r[-1] < 0.2 * r[0]


def test_golden_vectors():
    """Regression pins of the oracle (generated by tests/golden/make_golden.py)."""
    path = os.path.join(ROOT, "tests", "golden", "bump_17x9x9.npz")
    g = np.load(path)
    blk, prm, fs = case.bump_case(17, 9, 9)
    o = Oracle(blk, prm)
    o.start()
    o.statim(); o.adjuin(); o.residu(1, 1)
    for n in ("DRO", "DM", "DN", "DW", "DE"):
        np.testing.assert_allclose(interior(blk, blk.arrays[n]), g["res_" + n], rtol=1e-13,
                                   atol=1e-13 * np.abs(g["res_" + n]).max())
    hist = np.array([o.cycle(i + 1)[0] for i in range(10)])
    np.testing.assert_allclose(hist, g["hist10"], rtol=1e-11)


def test_abi_exports_every_declared_symbol():
    """libfinflo_gpu.so loads without a GPU and exports every function that
    include/finflo_gpu.h declares."""
    from finflo_b200 import gpu
    gpu.build()
    L = ctypes.CDLL(gpu.LIB_PATH)
    hdr = open(os.path.join(ROOT, "include", "finflo_gpu.h")).read()
    names = re.findall(r"^\s*(?:int|void \*|const char \*)\s*\**\s*(ff_\w+)\s*\(", hdr, re.M)
    assert len(names) >= 15
    # the Fortran call-site wrappers: gfortran names (lower case, trailing _)
    fnames = re.findall(r"^\s*void\s+([a-z]+_)\s*\(", hdr, re.M)
    assert sorted(fnames) == ["boundi_", "fin_", "impsdi_", "residi_", "statim_"]
    for n in names + fnames:
        assert hasattr(L, n), n
    assert L.ff_abi_version() == 7


def test_nn_abi_exports_every_declared_symbol():
    """libfinflo_nn.so (the warm start's tensor-core kernels) loads without a
    GPU and exports every function that include/finflo_nn.h declares."""
    from finflo_b200 import nn
    nn.build()
    L = ctypes.CDLL(nn.LIB_PATH)
    hdr = open(os.path.join(ROOT, "include", "finflo_nn.h")).read()
    names = re.findall(r"^\s*int\s+(ffnn_\w+)\s*\(", hdr, re.M)
    assert sorted(names) == sorted(nn.SYMBOLS)
    for n in names:
        assert hasattr(L, n), n


@pytest.mark.parametrize("flux", [f for f in case.FLUX if f != "roe"])
def test_flux_scheme_oracle_converges(flux):
    """Whole laminar cycles with each IFLUX scheme besides Roe: finite, the
    residual falls two decades in 60 cycles.  AUSM runs the slip-wall
    channel at CFL 1: as FLUXAU is written, its momentum flux carries PDIFF
    while BOTSKE's wall pressure stays P (YP1 = 1 for IFLUX = 3,
    base3c.f:6304-6315), so a no-slip wall leaves FRSPRE * A on its cells,
    and the pressure work of its energy flux is the unsplit central
    average; there the residual falls, then grows again after ~70 cycles."""
    if flux == "ausm":
        blk, prm, fs = case.bump_case(17, 9, 9, cfl=1.0)
        for pa in blk.patches:
            if pa.ityp == grid.BC_SOL:
                pa.ityp = grid.BC_MIR
        prm.idi1 = prm.idi2 = prm.idi3 = 0
        prm.fullns = 0
    else:
        blk, prm, fs = case.bump_case(17, 9, 9)
    prm.flux = case.FLUX[flux]
    o = Oracle(blk, prm)
    o.start()
    r = np.array([o.cycle(i + 1)[0][0] for i in range(60)])
    assert np.isfinite(r).all()
    assert r[-1] < 0.01 * r[0]
