"""Block geometry in the FINFLO storage layout (set-up only, not on the hot path).

A block is stored as linear FP64 arrays with two ghost layers on every side
(``IN=JN=KN=2``, charac.f:179), i fastest.  With ``ISTRID = IMAX+4`` and
``IL = ISTRID*(JMAX+4)`` the 0-based storage index of the 1-based cell
(I, J, K) is ``(K+1)*IL + (J+1)*ISTRID + (I+1)`` (res3c.f:127-136,
ns3c.f:2419 for the per-block offsets).

Face arrays follow the reference convention: ``A1(N)``/``A1XA(N)``... hold the
area and unit normal of the i-face on the LOW side of cell N (the face between
N-1 and N), pointing towards +i; likewise A2 (j) and A3 (k).  ``D1..D3`` are
the cell thicknesses of D1D2D3 (gluebm.f:2326-2372):
``min(1e4, (V+eps)/(A_low+A_high+eps)*2)``.

The grid metrics themselves (GRIVAL/AREVC1, ns3c.f:5636, gluebm.f:1586) are not
restated: this module computes them from node coordinates with the
diagonal-cross-product face vectors, so every cell is exactly closed
(sum of outward face vectors = 0) and ghost cells get the geometry of
mirror-extrapolated ghost nodes.  The oracle and the CUDA path both take the
metrics as inputs, so parity does not depend on how they were produced.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

NG = 2  # ghost layers per side (IN = JN = KN = 2)

# ICON(1) boundary types (gluebm.f:2737-2797)
BC_INL = 3
BC_MIR = 4
BC_OUT = 5
BC_SOL = 8
BC_CON = 1


def strides(imax: int, jmax: int, kmax: int):
    istrid = imax + 2 * NG
    jstrid = jmax + 2 * NG
    kstrid = kmax + 2 * NG
    return istrid, istrid * jstrid, istrid * jstrid * kstrid


def sidx(i, j, k, imax, jmax):
    """0-based storage index of 1-based cell (i, j, k) (ghosts: 0, -1, MAX+1, MAX+2)."""
    istrid = imax + 2 * NG
    il = istrid * (jmax + 2 * NG)
    return (k + 1) * il + (j + 1) * istrid + (i + 1)


def tanh_stretch(n_cells: int, h1: float) -> np.ndarray:
    """One-sided tanh distribution on [0,1] with first-cell height ``h1``."""
    eta = np.linspace(0.0, 1.0, n_cells + 1)

    def first(delta):
        return 1.0 + math.tanh(delta * (1.0 / n_cells - 1.0)) / math.tanh(delta)

    lo, hi = 1e-6, 50.0
    if first(lo) <= h1:
        return eta
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if first(mid) > h1:
            lo = mid
        else:
            hi = mid
    delta = 0.5 * (lo + hi)
    return 1.0 + np.tanh(delta * (eta - 1.0)) / math.tanh(delta)


def bump_nodes(ni: int, nj: int, nk: int, h1: float = 1e-3, amp: float = 0.1,
               xlen: float = 3.0, zlen: float = 0.5, span_amp: float = 0.0,
               x0: float = 0.0, y_top: float = 1.0):
    """Node coordinates (nk, nj, ni) of the bump channel.

    Lower wall ``y = a(z)*sin^2(pi(x-1))`` on 1<=x<=2, else 0, with
    ``a(z) = amp*(1 + span_amp*sin(2 pi z))``; top wall ``y = y_top``;
    uniform in x and z, tanh-stretched in y with first-cell height ``h1``.
    """
    x = x0 + np.linspace(0.0, xlen, ni)
    z = np.linspace(0.0, zlen, nk)
    s = tanh_stretch(nj - 1, h1)
    X = np.empty((nk, nj, ni))
    Y = np.empty_like(X)
    Z = np.empty_like(X)
    for k in range(nk):
        a = amp * (1.0 + span_amp * math.sin(2.0 * math.pi * z[k]))
        yb = np.where((x >= 1.0) & (x <= 2.0), a * np.sin(np.pi * (x - 1.0)) ** 2, 0.0)
        for j in range(nj):
            X[k, j, :] = x
            Y[k, j, :] = yb + (y_top - yb) * s[j]
            Z[k, j, :] = z[k]
    return X, Y, Z


def box_nodes(x, y, z):
    """Cartesian tensor-product nodes from 1-D coordinate vectors."""
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    return X.copy(), Y.copy(), Z.copy()


def _extend(a: np.ndarray, ng: int = NG) -> np.ndarray:
    """Add ng ghost node layers per side by mirror extrapolation x[-m] = 2x[0]-x[m]."""
    for ax in range(3):
        n = a.shape[ax]
        lo = [2 * np.take(a, 0, axis=ax) - np.take(a, m, axis=ax) for m in range(ng, 0, -1)]
        hi = [2 * np.take(a, n - 1, axis=ax) - np.take(a, n - 1 - m, axis=ax) for m in range(1, ng + 1)]
        a = np.concatenate([np.expand_dims(t, ax) for t in lo] + [a]
                           + [np.expand_dims(t, ax) for t in hi], axis=ax)
    return a


@dataclass
class Metrics:
    imax: int
    jmax: int
    kmax: int
    arrays: dict = field(default_factory=dict)

    @property
    def ntot(self):
        return strides(self.imax, self.jmax, self.kmax)[2]


METRIC_NAMES = ("A1", "A1XA", "A1YA", "A1ZA", "A2", "A2XA", "A2YA", "A2ZA",
                "A3", "A3XA", "A3YA", "A3ZA", "VOL", "XC", "YC", "ZC",
                "D1", "D2", "D3")


def compute_metrics(X, Y, Z, ng: int = NG, raw: bool = False):
    """Metrics of all cells (ng ghost layers) from interior node arrays (nk,nj,ni)."""
    nk, nj, ni = X.shape
    imax, jmax, kmax = ni - 1, nj - 1, nk - 1
    P = np.stack([_extend(X, ng), _extend(Y, ng), _extend(Z, ng)], axis=-1)
    ks, js, is_ = kmax + 2 * ng, jmax + 2 * ng, imax + 2 * ng

    def face_vec(c00, c11, c01, c10):
        return 0.5 * np.cross(c11 - c00, c01 - c10)

    # i-faces on the low side of storage (s,t,u): node plane s
    p = P
    Si = face_vec(p[:ks, :js, :is_], p[1:ks + 1, 1:js + 1, :is_],
                  p[1:ks + 1, :js, :is_], p[:ks, 1:js + 1, :is_])
    Sj = face_vec(p[:ks, :js, :is_], p[1:ks + 1, :js, 1:is_ + 1],
                  p[:ks, :js, 1:is_ + 1], p[1:ks + 1, :js, :is_])
    Sk = face_vec(p[:ks, :js, :is_], p[:ks, 1:js + 1, 1:is_ + 1],
                  p[:ks, 1:js + 1, :is_], p[:ks, :js, 1:is_ + 1])
    # high-side faces needed for the volume / D arrays
    Si_hi = face_vec(p[:ks, :js, 1:is_ + 1], p[1:ks + 1, 1:js + 1, 1:is_ + 1],
                     p[1:ks + 1, :js, 1:is_ + 1], p[:ks, 1:js + 1, 1:is_ + 1])
    Sj_hi = face_vec(p[:ks, 1:js + 1, :is_], p[1:ks + 1, 1:js + 1, 1:is_ + 1],
                     p[:ks, 1:js + 1, 1:is_ + 1], p[1:ks + 1, 1:js + 1, :is_])
    Sk_hi = face_vec(p[1:ks + 1, :js, :is_], p[1:ks + 1, 1:js + 1, 1:is_ + 1],
                     p[1:ks + 1, 1:js + 1, :is_], p[1:ks + 1, :js, 1:is_ + 1])

    def centroid(a, b, c, d):
        return 0.25 * (a + b + c + d)

    ci_lo = centroid(p[:ks, :js, :is_], p[1:ks + 1, :js, :is_], p[:ks, 1:js + 1, :is_], p[1:ks + 1, 1:js + 1, :is_])
    ci_hi = centroid(p[:ks, :js, 1:is_ + 1], p[1:ks + 1, :js, 1:is_ + 1], p[:ks, 1:js + 1, 1:is_ + 1], p[1:ks + 1, 1:js + 1, 1:is_ + 1])
    cj_lo = centroid(p[:ks, :js, :is_], p[1:ks + 1, :js, :is_], p[:ks, :js, 1:is_ + 1], p[1:ks + 1, :js, 1:is_ + 1])
    cj_hi = centroid(p[:ks, 1:js + 1, :is_], p[1:ks + 1, 1:js + 1, :is_], p[:ks, 1:js + 1, 1:is_ + 1], p[1:ks + 1, 1:js + 1, 1:is_ + 1])
    ck_lo = centroid(p[:ks, :js, :is_], p[:ks, 1:js + 1, :is_], p[:ks, :js, 1:is_ + 1], p[:ks, 1:js + 1, 1:is_ + 1])
    ck_hi = centroid(p[1:ks + 1, :js, :is_], p[1:ks + 1, 1:js + 1, :is_], p[1:ks + 1, :js, 1:is_ + 1], p[1:ks + 1, 1:js + 1, 1:is_ + 1])

    vol = (np.sum(ci_hi * Si_hi, -1) - np.sum(ci_lo * Si, -1)
           + np.sum(cj_hi * Sj_hi, -1) - np.sum(cj_lo * Sj, -1)
           + np.sum(ck_hi * Sk_hi, -1) - np.sum(ck_lo * Sk, -1)) / 3.0
    cen = 0.125 * sum(p[a:a + ks, b:b + js, c:c + is_] for a in (0, 1) for b in (0, 1) for c in (0, 1))

    out = {}
    for name, S in (("A1", Si), ("A2", Sj), ("A3", Sk)):
        mag = np.sqrt(np.sum(S * S, -1))
        safe = np.where(mag > 0, mag, 1.0)
        out[name] = mag
        out[name + "XA"] = S[..., 0] / safe
        out[name + "YA"] = S[..., 1] / safe
        out[name + "ZA"] = S[..., 2] / safe
    out["VOL"] = vol
    out["XC"], out["YC"], out["ZC"] = cen[..., 0], cen[..., 1], cen[..., 2]
    eps = 1e-20
    a1h = np.sqrt(np.sum(Si_hi * Si_hi, -1))
    a2h = np.sqrt(np.sum(Sj_hi * Sj_hi, -1))
    a3h = np.sqrt(np.sum(Sk_hi * Sk_hi, -1))
    out["D1"] = np.minimum(1e4, (vol + eps) / (out["A1"] + a1h + eps) * 2.0)
    out["D2"] = np.minimum(1e4, (vol + eps) / (out["A2"] + a2h + eps) * 2.0)
    out["D3"] = np.minimum(1e4, (vol + eps) / (out["A3"] + a3h + eps) * 2.0)
    if raw:
        return dict(S1=Si, S2=Sj, S3=Sk, S1h=Si_hi, S2h=Sj_hi, S3h=Sk_hi, VOL=vol, C=cen,
                    dims=(imax, jmax, kmax), ng=ng)
    m = Metrics(imax, jmax, kmax)
    for k2 in METRIC_NAMES:
        m.arrays[k2] = np.ascontiguousarray(out[k2], dtype=np.float64).reshape(-1)
    return m


def _finish(S1, S2, S3, S1h, S2h, S3h, vol, cen, dims, ng):
    """Metrics arrays (2 ghost layers) from face vectors, volumes and centres
    given with ng >= 2 ghost layers."""
    imax, jmax, kmax = dims
    c = ng - NG
    sl = (slice(c, c + kmax + 2 * NG), slice(c, c + jmax + 2 * NG), slice(c, c + imax + 2 * NG))
    out = {}
    for name, S in (("A1", S1), ("A2", S2), ("A3", S3)):
        S = S[sl]
        mag = np.sqrt(np.sum(S * S, -1))
        safe = np.where(mag > 0, mag, 1.0)
        out[name] = mag
        out[name + "XA"] = S[..., 0] / safe
        out[name + "YA"] = S[..., 1] / safe
        out[name + "ZA"] = S[..., 2] / safe
    v = vol[sl]
    out["VOL"] = v
    cc = cen[sl]
    out["XC"], out["YC"], out["ZC"] = cc[..., 0], cc[..., 1], cc[..., 2]
    eps = 1e-20
    for d, Sh in (("1", S1h), ("2", S2h), ("3", S3h)):
        ah = np.sqrt(np.sum(Sh[sl] ** 2, -1))
        out["D" + d] = np.minimum(1e4, (v + eps) / (out["A" + d] + ah + eps) * 2.0)
    m = Metrics(imax, jmax, kmax)
    for k2 in METRIC_NAMES:
        m.arrays[k2] = np.ascontiguousarray(out[k2], dtype=np.float64).reshape(-1)
    return m


def _lump(r):
    """One coarsening step (GRID1B/LUMPA1 gluebm.f:1492-1496): coarse volumes
    are sums of the 8 children, coarse face vectors sums of the 4 child
    faces, centres volume-weighted; ng halves."""
    ng = r["ng"]
    imax, jmax, kmax = r["dims"]
    assert ng % 2 == 0 and imax % 2 == 0 and jmax % 2 == 0 and kmax % 2 == 0
    vol, cen = r["VOL"], r["C"]

    def csum(a):  # sum over 2x2x2 children (k, j, i axes)
        return (a[0::2, 0::2, 0::2] + a[0::2, 0::2, 1::2] + a[0::2, 1::2, 0::2] + a[0::2, 1::2, 1::2]
                + a[1::2, 0::2, 0::2] + a[1::2, 0::2, 1::2] + a[1::2, 1::2, 0::2] + a[1::2, 1::2, 1::2])
    vc = csum(vol)
    cc = csum(cen * vol[..., None]) / vc[..., None]
    S1 = r["S1"][0::2, 0::2, 0::2] + r["S1"][0::2, 1::2, 0::2] + r["S1"][1::2, 0::2, 0::2] + r["S1"][1::2, 1::2, 0::2]
    S2 = r["S2"][0::2, 0::2, 0::2] + r["S2"][0::2, 0::2, 1::2] + r["S2"][1::2, 0::2, 0::2] + r["S2"][1::2, 0::2, 1::2]
    S3 = r["S3"][0::2, 0::2, 0::2] + r["S3"][0::2, 0::2, 1::2] + r["S3"][0::2, 1::2, 0::2] + r["S3"][0::2, 1::2, 1::2]
    S1h = r["S1h"][0::2, 0::2, 1::2] + r["S1h"][0::2, 1::2, 1::2] + r["S1h"][1::2, 0::2, 1::2] + r["S1h"][1::2, 1::2, 1::2]
    S2h = r["S2h"][0::2, 1::2, 0::2] + r["S2h"][0::2, 1::2, 1::2] + r["S2h"][1::2, 1::2, 0::2] + r["S2h"][1::2, 1::2, 1::2]
    S3h = r["S3h"][1::2, 0::2, 0::2] + r["S3h"][1::2, 0::2, 1::2] + r["S3h"][1::2, 1::2, 0::2] + r["S3h"][1::2, 1::2, 1::2]
    return dict(S1=S1, S2=S2, S3=S3, S1h=S1h, S2h=S2h, S3h=S3h, VOL=vc, C=cc,
                dims=(imax // 2, jmax // 2, kmax // 2), ng=ng // 2)


def mg_metrics(X, Y, Z, nlev: int):
    """Metrics of every multigrid level (level 1 first), coarse levels
    lumped from the fine cells so that the 8 children of a coarse cell fill
    it exactly (volumes and face vectors add up)."""
    ng = NG * 2 ** (nlev - 1)
    r = compute_metrics(X, Y, Z, ng=ng, raw=True)
    levels = []
    for lev in range(nlev):
        levels.append(_finish(r["S1"], r["S2"], r["S3"], r["S1h"], r["S2h"], r["S3h"], r["VOL"], r["C"],
                              r["dims"], r["ng"]))
        if lev + 1 < nlev:
            r = _lump(r)
    return levels
