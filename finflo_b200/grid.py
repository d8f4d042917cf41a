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

The metrics follow the reference's set-up (GRIVAL ns3c.f:5636 -> GRID1B
gluebm.f:1265): ghost nodes as GRIDEX (1029), face areas, unit normals,
volumes (three passes) and centres as AREVC1 (1586), thicknesses as D1D2D3
(2326), coarse levels as LUMPA1 / LUMPVS (2194, 2256), in the reference's
order of operations, so that the interior cells, their faces and the first
ghost layer equal the reference's to the bit.  The further ghost layers (the
reference fills them in BOUNDX / BOUNDV / MIRC / CONEC after GRID1B) come
from continued mirror reflection of the nodes and, on coarse levels, from
lumping the fine ghost cells.
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
    """Add ng ghost node layers per side.  The first layer is GRIDEX's
    (gluebm.f:1029, REFXYZ 1175): faces reflected, x[-1] = 2 x[0] - x[1],
    and the edges and corners reflected diagonally through the first
    interior node, x[-1, -1] = 2 x[0, 0] - x[1, 1].  Further layers (the
    reference keeps one) continue the mirror reflection along each axis in
    turn, x[-m] = 2 x[0] - x[m]."""
    for ax in range(3):
        n = a.shape[ax]
        lo = [2 * np.take(a, 0, axis=ax) - np.take(a, m, axis=ax) for m in range(ng, 0, -1)]
        hi = [2 * np.take(a, n - 1, axis=ax) - np.take(a, n - 1 - m, axis=ax) for m in range(1, ng + 1)]
        a = np.concatenate([np.expand_dims(t, ax) for t in lo] + [a]
                           + [np.expand_dims(t, ax) for t in hi], axis=ax)
    if ng >= 1:
        _gridex_edges(a, ng)
    return a


def _gridex_edges(e: np.ndarray, ng: int):
    """GRIDEX's diagonal reflection of the first-layer edge and corner nodes
    of the extended array e (ng layers), in place."""
    n = [e.shape[ax] - 2 * ng for ax in range(3)]

    def pos(ax, side):   # (ghost, first interior, second interior) indices
        return (ng - 1, ng, ng + 1) if side == 0 else (ng + n[ax], ng + n[ax] - 1, ng + n[ax] - 2)

    for u, v in ((0, 1), (0, 2), (1, 2)):        # edges: two ghost axes, the third interior
        w = 3 - u - v
        for su in (0, 1):
            for sv in (0, 1):
                pu, pv = pos(u, su), pos(v, sv)
                idx, src1, src2 = [None] * 3, [None] * 3, [None] * 3
                idx[u], idx[v], idx[w] = pu[0], pv[0], slice(ng, ng + n[w])
                src1[u], src1[v], src1[w] = pu[1], pv[1], slice(ng, ng + n[w])
                src2[u], src2[v], src2[w] = pu[2], pv[2], slice(ng, ng + n[w])
                e[tuple(idx)] = 2. * e[tuple(src1)] - e[tuple(src2)]
    for c in range(8):                           # corners
        p = [pos(ax, (c >> ax) & 1) for ax in range(3)]
        e[p[0][0], p[1][0], p[2][0]] = 2. * e[p[0][1], p[1][1], p[2][1]] - e[p[0][2], p[1][2], p[2][2]]


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


# AREVC1's corner nodes of a cell in its pass for direction d (0 = i, 1 = j,
# 2 = k): the pass's (ISTR, JSTR, KSTR) are the axes (d, d+1, d+2) cyclic,
# and the corners IT1..IT8 step by 0, KSTR, JSTR+KSTR, JSTR, ISTR,
# ISTR+KSTR, ISTR+JSTR+KSTR, ISTR+JSTR (gluebm.f:1640-1660).
def _corner_offsets(d):
    a, b, c = d, (d + 1) % 3, (d + 2) % 3
    steps = ((), (c,), (b, c), (b,), (a,), (a, c), (a, b, c), (a, b))
    out = []
    for st in steps:
        o = [0, 0, 0]
        for ax in st:
            o[ax] = 1
        out.append(tuple(o))   # (di, dj, dk)
    return out


def _arevc1(P, ncell):
    """AREVC1 gluebm.f:1586 on the extended nodes P [k, j, i, 3] for every
    cell of the ncell = (ci, cj, ck) storage range: per direction the face
    vectors (AXX, AYY, AZZ) of the ncell[d] + 1 face planes, and the cell
    volumes accumulated over the three passes (VSUM, VDIV) and the centres
    of the last pass."""
    ci, cj, ck = ncell
    faces, vol, cen = [], None, None
    for d in range(3):
        nf = [ci, cj, ck]
        nf[d] += 1
        offs = _corner_offsets(d)

        def corner(q, nrange):
            di, dj, dk = offs[q]
            return P[dk:dk + nrange[2], dj:dj + nrange[1], di:di + nrange[0]]

        # face vectors of the face planes 0..ncell[d] (IT0 form, corners 1-4)
        p1, p2, p3, p4 = (corner(q, nf) for q in range(4))
        x1, y1, z1 = p1[..., 0], p1[..., 1], p1[..., 2]
        x2, y2, z2 = p2[..., 0], p2[..., 1], p2[..., 2]
        x3, y3, z3 = p3[..., 0], p3[..., 1], p3[..., 2]
        x4, y4, z4 = p4[..., 0], p4[..., 1], p4[..., 2]
        axx = 0.5 * ((z3 - z1) * (y4 - y2) - (y3 - y1) * (z4 - z2))
        ayy = 0.5 * ((x3 - x1) * (z4 - z2) - (z3 - z1) * (x4 - x2))
        azz = 0.5 * ((y3 - y1) * (x4 - x2) - (x3 - x1) * (y4 - y2))
        faces.append(np.stack([axx, ayy, azz], axis=-1))
        # the cell terms of the pass: centre, diagonals, low and high face
        c = [corner(q, ncell) for q in range(8)]
        xce = 0.125 * (c[0] + c[1] + c[2] + c[3] + c[4] + c[5] + c[6] + c[7])
        rd = xce - 0.5 * (c[0] + c[1])
        rd2 = xce - 0.5 * (c[6] + c[7])
        sl_lo = [slice(0, ck), slice(0, cj), slice(0, ci)]
        sl_hi = list(sl_lo)
        sl_hi[2 - d] = slice(1, ncell[d] + 1)
        lo = faces[d][tuple(sl_lo)]
        hi = -faces[d][tuple(sl_hi)]                 # AXX2 = -(next cell's AXX)
        # (VSUM V + RDIAG.A + RD2AG.A2) / VDIV, summed left to right
        v = np.zeros(lo.shape[:-1]) if d == 0 else vol
        for t in (rd[..., 0] * lo[..., 0], rd[..., 1] * lo[..., 1], rd[..., 2] * lo[..., 2],
                  rd2[..., 0] * hi[..., 0], rd2[..., 1] * hi[..., 1], rd2[..., 2] * hi[..., 2]):
            v = v + t
        vol = v / 3.0 if d == 2 else v
        cen = xce
    return faces, vol, cen


def _area_normal(S):
    """AREVC1's area A = sqrt(AXX**2 + AYY**2 + AZZ**2) and unit normal
    A*/(A + 1e-20); a zero-area face keeps the normal (1, 0, 0)."""
    a = np.sqrt(S[..., 0] * S[..., 0] + S[..., 1] * S[..., 1] + S[..., 2] * S[..., 2])
    n = S / (a + 1.0e-20)[..., None]
    z = a < 1.0e-20
    n[z] = (1.0, 0.0, 0.0)
    return a, n


def compute_metrics(X, Y, Z, ng: int = NG, raw: bool = False):
    """Metrics of all cells (ng ghost layers) from interior node arrays
    (nk, nj, ni), by AREVC1 on the GRIDEX-extended nodes; D1..D3 as
    D1D2D3 (gluebm.f:2326)."""
    nk, nj, ni = X.shape
    imax, jmax, kmax = ni - 1, nj - 1, nk - 1
    P = np.stack([_extend(X, ng), _extend(Y, ng), _extend(Z, ng)], axis=-1)
    ncell = (imax + 2 * ng, jmax + 2 * ng, kmax + 2 * ng)
    faces, vol, cen = _arevc1(P, ncell)
    r = dict(dims=(imax, jmax, kmax), ng=ng, VOL=vol, C=cen)
    for d in range(3):
        r[f"A{d + 1}"], r[f"N{d + 1}"] = _area_normal(faces[d])
    if raw:
        return r
    return _finish(r)


def _finish(r):
    """Metrics arrays (2 ghost layers) from per-face areas and normals
    (one more face plane than cells in each face's direction), volumes and
    centres given with ng >= 2 ghost layers."""
    imax, jmax, kmax = r["dims"]
    ng = r["ng"]
    c = ng - NG
    ks, js, is_ = kmax + 2 * NG, jmax + 2 * NG, imax + 2 * NG
    sl = (slice(c, c + ks), slice(c, c + js), slice(c, c + is_))
    out = {}
    v = r["VOL"][sl]
    out["VOL"] = v
    cc = r["C"][sl]
    out["XC"], out["YC"], out["ZC"] = cc[..., 0], cc[..., 1], cc[..., 2]
    eps = 1e-20
    for d in range(3):
        A, N = r[f"A{d + 1}"], r[f"N{d + 1}"]
        name = f"A{d + 1}"
        out[name] = A[sl]
        out[name + "XA"] = N[sl][..., 0]
        out[name + "YA"] = N[sl][..., 1]
        out[name + "ZA"] = N[sl][..., 2]
        hs = list(sl)
        hs[2 - d] = slice(sl[2 - d].start + 1, sl[2 - d].stop + 1)
        out[f"D{d + 1}"] = np.minimum(1e4, (v + eps) / (A[sl] + A[tuple(hs)] + eps) * 2.0)
    m = Metrics(imax, jmax, kmax)
    for k2 in METRIC_NAMES:
        m.arrays[k2] = np.ascontiguousarray(out[k2], dtype=np.float64).reshape(-1)
    return m


def _lump(r):
    """One coarsening step: LUMPA1 gluebm.f:2194 for the faces (area = sum
    of the four child areas + 1e-20, normal = the area-weighted sum of the
    child normals, normalised; (1, ., .) where that sum vanishes) and LUMPVS
    gluebm.f:2256 for volumes and volume-weighted centres, children in the
    reference's order (i, j, k), (i, j+1, k), (i, j, k+1), (i, j+1, k+1),
    then the same at i+1; ghost layers halve."""
    ng = r["ng"]
    imax, jmax, kmax = r["dims"]
    assert ng % 2 == 0 and imax % 2 == 0 and jmax % 2 == 0 and kmax % 2 == 0
    vol, cen = r["VOL"], r["C"]
    ck, cj, ci = (n // 2 for n in vol.shape)

    def child(a, di, dj, dk):
        return a[dk::2, dj::2, di::2][:ck, :cj, :ci]

    order = [(0, 0, 0), (0, 1, 0), (0, 0, 1), (0, 1, 1), (1, 0, 0), (1, 1, 0), (1, 0, 1), (1, 1, 1)]
    vs = [child(vol, *o) for o in order]
    vl = vs[0]
    for q in range(1, 8):
        vl = vl + vs[q]
    cs = [child(cen, *o) for o in order]
    s = vs[0][..., None] * cs[0]
    for q in range(1, 8):
        s = s + vs[q][..., None] * cs[q]
    out = dict(dims=(imax // 2, jmax // 2, kmax // 2), ng=ng // 2, VOL=vl, C=s / vl[..., None])
    for d in range(3):
        A, N = r[f"A{d + 1}"], r[f"N{d + 1}"]
        nf = [ci, cj, ck]
        nf[d] += 1
        bd, cd = (d + 1) % 3, (d + 2) % 3           # LUMPA1's J and K directions of the pass
        kids = []
        for q in range(4):
            o = [0, 0, 0]
            if q & 1:
                o[bd] = 1
            if q & 2:
                o[cd] = 1
            sl = tuple(slice(o[ax], o[ax] + 2 * nf[ax], 2) for ax in (2, 1, 0))
            kids.append((A[sl], N[sl]))
        vec = kids[0][0][..., None] * kids[0][1]
        for q in range(1, 4):
            vec = vec + kids[q][0][..., None] * kids[q][1]
        al = kids[0][0] + kids[1][0] + kids[2][0] + kids[3][0] + 1.0e-20
        axyzl = np.sqrt(vec[..., 0] * vec[..., 0] + vec[..., 1] * vec[..., 1] + vec[..., 2] * vec[..., 2])
        n = vec / (axyzl + 1.0e-20)[..., None]
        z = axyzl < 1.0e-20
        n[..., 0] = np.where(z, 1.0, n[..., 0])
        out[f"A{d + 1}"], out[f"N{d + 1}"] = al, n
    return out


def mg_metrics(X, Y, Z, nlev: int):
    """Metrics of every multigrid level (level 1 first), coarse levels
    lumped from the fine cells (LUMPA1 / LUMPVS); the ghost layers of a
    coarse level are lumped from the fine level's, which carries
    2 * 2^(nlev-1) of them."""
    ng = NG * 2 ** (nlev - 1)
    r = compute_metrics(X, Y, Z, ng=ng, raw=True)
    levels = []
    for lev in range(nlev):
        levels.append(_finish(r))
        if lev + 1 < nlev:
            r = _lump(r)
    return levels
