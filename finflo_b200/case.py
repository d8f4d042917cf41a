"""Case set-up: block geometry, boundary patches, constants and initial state.

Everything here runs once on the host before the iteration loop (the
reference's INPUT/READBC/INIT/GRIVAL stage, main.f:1210, gluebm.f:2553,
ns3c.f:4360, 5636).  The arrays are laid out exactly as the reference stores a
block (two ghost layers, i fastest) so they can be handed to the device
library or to a FINFLO host unchanged.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field

import numpy as np

from . import grid

# ---- C structs shared with the library (include/finflo_types.h) ----------


class FFPatch(ctypes.Structure):
    _fields_ = [("ityp", ctypes.c_int), ("iface", ctypes.c_int),
                ("r1a", ctypes.c_int), ("r1b", ctypes.c_int),
                ("r2a", ctypes.c_int), ("r2b", ctypes.c_int),
                ("ibtype", ctypes.c_int), ("iheat", ctypes.c_int),
                ("nface", ctypes.c_int), ("iori", ctypes.c_int),
                ("n1a", ctypes.c_int), ("n2a", ctypes.c_int),
                ("bounr", ctypes.c_double), ("bounu", ctypes.c_double),
                ("bounv", ctypes.c_double), ("bounw", ctypes.c_double),
                ("bount", ctypes.c_double), ("bounp", ctypes.c_double),
                ("bounpd", ctypes.c_double), ("bounrk", ctypes.c_double),
                ("bounep", ctypes.c_double)]


class FFParams(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in (
        "gamma", "rgas", "pr", "prt", "visu0", "expsu", "tsu0", "e0ref", "t0ref",
        "frsden", "frspre", "frsvel", "frsvis", "frstem", "cfl", "cfll", "theta",
        "cdiff", "pvisc", "tlolim", "tuplim", "cmgk", "cmgeps",
        "rklim", "epslim", "turlim", "csimps", "re")] + [
        (n, ctypes.c_int) for n in (
            "interi", "interj", "interk", "entropy_fix", "iturb", "fullns",
            "idi1", "idi2", "idi3", "coarse_inter", "lusgs_fp32", "ddadi", "timel", "flux")] + [
        ("dt", ctypes.c_double), ("predgs_full", ctypes.c_int), ("res_fp32", ctypes.c_int),
        ("xxtral", ctypes.c_int), ("rjk2", ctypes.c_double), ("rjk4", ctypes.c_double)]


class FFHaloItem(ctypes.Structure):
    """ff_halo_item of include/finflo_gpu.h."""
    _fields_ = [("blk", ctypes.c_int), ("mode", ctypes.c_int), ("offset", ctypes.c_longlong),
                ("pa", FFPatch)]


# enum ff_slot (include/finflo_types.h), in order
SLOTS = ["RO", "RM", "RN", "RW", "E", "P", "PDIFF", "U", "V", "W", "C",
         "TEMP", "VIS", "CH", "CP", "DRDP", "DRDH", "EPS2", "VIST",
         "DRO", "DM", "DN", "DW", "DE", "DRK", "DEPS", "DTL",
         "TOLD", "UOLD", "VOLD", "WOLD", "POLD",
         "A1", "A1XA", "A1YA", "A1ZA", "A2", "A2XA", "A2YA", "A2ZA",
         "A3", "A3XA", "A3YA", "A3ZA", "VOL", "XC", "YC", "ZC", "D1", "D2", "D3",
         "W12", "W13", "W23", "S11", "S12", "S13", "S22", "S23", "S33",
         "DTDX", "DTDY", "DTDZ", "OHMI", "STRAIN",
         "F1R", "F1RM", "F1RN", "F1RW", "F1E",
         "ROP2H", "RMP2H", "RNP2H", "RWP2H", "EP2H",
         "RK", "REPS", "DISTW", "FUN1", "SRK", "SEPS", "PTUR",
         "DKDX", "DKDY", "DKDZ", "DEDX", "DEDY", "DEDZ",
         "RKOLD", "EPSOLD", "F1RK", "F1EPS", "RKP2H", "EPP2H",
         "ROLE2", "RMLE2", "RNLE2", "RWLE2", "ELE2", "RKLE2", "EPSLE2",
         "ROLE3", "RMLE3", "RNLE3", "RWLE3", "ELE3", "RKLE3", "EPSLE3",
         "SCALEJ"]
SLOT = {n: i for i, n in enumerate(SLOTS)}
STATE_SLOTS = SLOTS[:19]
METRIC_SLOTS = list(grid.METRIC_NAMES)


@dataclass
class FlowConditions:
    mach: float = 0.5
    reynolds: float = 1.0e4          # per unit length
    temperature: float = 288.15      # FRSTEM [K]
    gamma: float = 1.4
    rgas: float = 287.05287
    pr: float = 0.72
    prt: float = 0.9
    visu0: float = 1.458e-6
    expsu: float = 1.5
    tsu0: float = 110.4

    def freestream(self):
        t = self.temperature
        c = math.sqrt(self.gamma * self.rgas * t)
        u = self.mach * c
        mu = self.visu0 * t * math.sqrt(t) / (t + self.tsu0)
        if self.reynolds > 0:
            rho = self.reynolds * mu / u
        else:
            rho = 1.2
        p = rho * self.rgas * t
        return dict(rho=rho, u=u, p=p, t=t, mu=mu, c=c)


# enum ff_flux (include/finflo_types.h): the inviscid face flux by the
# reference's FLUXTY names (FLUXME multi.f:3567)
FLUX = {"roe": 0, "vanleer": 1, "wps": 2, "ausm": 3, "kt": 7, "hcusp": 8}
FLUX_LAMINAR_ONLY = ("vanleer", "wps", "ausm")   # no RESIKE form (res3c.f:6946-7030)


def make_params(fc: FlowConditions, dims, *, cfl=2.0, cfll=2.0, inter=3,
                fullns=True, iturb=0, entropy_fix=False, lusgs_fp32=False, flux="roe") -> FFParams:
    fs = fc.freestream()
    p = FFParams()
    p.gamma, p.rgas, p.pr, p.prt = fc.gamma, fc.rgas, fc.pr, fc.prt
    p.visu0, p.expsu, p.tsu0 = fc.visu0, fc.expsu, fc.tsu0
    p.e0ref = p.t0ref = 0.0
    p.frsden, p.frspre, p.frsvel, p.frsvis, p.frstem = fs["rho"], fs["p"], fs["u"], fs["mu"], fs["t"]
    p.cfl, p.cfll = cfl, cfll
    p.theta, p.cdiff, p.pvisc = 1.5, 2.0, 1.8
    p.tlolim, p.tuplim = 0.05 * fs["t"], 6.0 * fs["t"]
    p.cmgk, p.cmgeps = 0.1, 0.2
    p.turlim, p.csimps = 5000.0, 5.0
    p.re = fs["rho"] * fs["u"] / fs["mu"]     # per unit reference length
    p.interi = p.interj = p.interk = inter
    p.entropy_fix = int(entropy_fix)
    p.iturb = iturb
    p.fullns = int(fullns)
    imax, jmax, kmax = dims
    # IDI1..3 default to the node counts (main.f:5657-5659): viscous everywhere
    p.idi1, p.idi2, p.idi3 = imax + 1, jmax + 1, kmax + 1
    p.coarse_inter = 55
    p.lusgs_fp32 = int(lusgs_fp32)
    p.flux = FLUX[flux]
    return p


def level_params(p: FFParams, level: int) -> FFParams:
    """IDM1..3 of a multigrid level (res3c.f:155-159, imps3.f:73-75)."""
    q = FFParams.from_buffer_copy(p)
    f = 2 ** (level - 1)
    q.idi1 = (p.idi1 - 1) // f + 1
    q.idi2 = (p.idi2 - 1) // f + 1
    q.idi3 = max(1, (p.idi3 - 1) // f) + 1 if p.idi3 != 0 else 0
    return q


@dataclass
class Block:
    imax: int
    jmax: int
    kmax: int
    arrays: dict
    patches: list
    nodes: tuple = None

    @property
    def dims(self):
        return self.imax, self.jmax, self.kmax

    @property
    def ntot(self):
        return grid.strides(self.imax, self.jmax, self.kmax)[2]

    @property
    def interior_cells(self):
        return self.imax * self.jmax * self.kmax

    def interior(self, name):
        a = self.arrays[name].reshape(self.kmax + 4, self.jmax + 4, self.imax + 4)
        return a[2:-2, 2:-2, 2:-2]

    def patch_array(self):
        arr = (FFPatch * max(1, len(self.patches)))()
        for i, pa in enumerate(self.patches):
            arr[i] = pa
        return arr


def _patch(ityp, iface, r1, r2, ibtype=0, iheat=0, **boun):
    pa = FFPatch()
    pa.ityp, pa.iface = ityp, iface
    pa.r1a, pa.r1b = r1
    pa.r2a, pa.r2b = r2
    pa.ibtype, pa.iheat = ibtype, iheat
    for k, v in boun.items():
        setattr(pa, k, v)
    return pa


def channel_patches(imax, jmax, kmax, fs, *, span="MIR"):
    """INL at i=1, OUT at i=IMAX, SOL lower/upper walls, MIR (or PER) spanwise."""
    inl = dict(bounr=fs["rho"], bounu=fs["u"], bounv=0.0, bounw=0.0, bount=fs["t"],
               bounp=fs["p"], bounpd=0.0)
    pats = [
        _patch(grid.BC_INL, 1, (1, jmax), (1, kmax), ibtype=4, **inl),
        _patch(grid.BC_OUT, 4, (1, jmax), (1, kmax), ibtype=3, **inl),
        _patch(grid.BC_SOL, 2, (1, imax), (1, kmax)),
        _patch(grid.BC_SOL, 5, (1, imax), (1, kmax)),
    ]
    if span == "MIR":
        pats += [_patch(grid.BC_MIR, 3, (1, imax), (1, jmax)),
                 _patch(grid.BC_MIR, 6, (1, imax), (1, jmax))]
    return pats


def new_block(X, Y, Z, patches) -> Block:
    m = grid.compute_metrics(X, Y, Z)
    ntot = m.ntot
    arrays = {n: np.zeros(ntot) for n in SLOTS}
    for n in METRIC_SLOTS:
        arrays[n][:] = m.arrays[n]
    return Block(m.imax, m.jmax, m.kmax, arrays, patches, nodes=(X, Y, Z))


def block_from_metrics(m, patches, nodes=None) -> Block:
    arrays = {n: np.zeros(m.ntot) for n in SLOTS}
    for n in METRIC_SLOTS:
        arrays[n][:] = m.arrays[n]
    return Block(m.imax, m.jmax, m.kmax, arrays, patches, nodes=nodes)


# ---- orientation of 1:1 patches (ICON(14)) ----------------------------------

# CORNER gluebm.f:2480: the four corner nodes of a patch, as (first, second)
# in-face node offsets from (lo, lo); odd faces go round the second index
# first, even faces the first.
_CORNER_ORDER = {1: ((0, 0), (0, 1), (1, 1), (1, 0)), 2: ((0, 0), (1, 0), (1, 1), (0, 1)),
                 3: ((0, 0), (0, 1), (1, 1), (1, 0)), 4: ((0, 0), (1, 0), (1, 1), (0, 1)),
                 5: ((0, 0), (0, 1), (1, 1), (1, 0)), 6: ((0, 0), (1, 0), (1, 1), (0, 1))}


def patch_corners(nodes, iface, r1, r2):
    """CORNER gluebm.f:2480: [4, 3] corner coordinates of the patch with cell
    ranges r1 = (r1a, r1b), r2 = (r2a, r2b) on face iface of the block with
    nodes (X, Y, Z), each [k, j, i]."""
    X, Y, Z = nodes
    kmax, jmax, imax = (n - 1 for n in X.shape)
    lo = (r1[0] - 1, r2[0] - 1)
    hi = (r1[1], r2[1])          # IXUQ + 1, IYUQ + 1 as 0-based node indices
    out = np.empty((4, 3))
    for q, (u, v) in enumerate(_CORNER_ORDER[iface]):
        t1 = hi[0] if u else lo[0]
        t2 = hi[1] if v else lo[1]
        d = (iface - 1) % 3
        layer = 0 if iface <= 3 else (imax, jmax, kmax)[d]
        i, j, k = (layer, t1, t2) if d == 0 else ((t1, layer, t2) if d == 1 else (t1, t2, layer))
        out[q] = X[k, j, i], Y[k, j, i], Z[k, j, i]
    return out


def orient(xcol, xcog, chlref=1.0):
    """ORIENT gluebm.f:8506: ICON(14) of a 1:1 patch from the diagonals of
    its corners xcol and its partner's xcog ([4, 3] each): the turn 0..3 of
    the partner whose diagonals match; -1 when none is within 1e-3 chlref."""
    a13, a24 = xcol[2] - xcol[0], xcol[3] - xcol[1]
    b13, b24 = xcog[2] - xcog[0], xcog[3] - xcog[1]
    b31, b42 = -b13, -b24
    nrm = np.linalg.norm
    s = [nrm(a13 - b13) + nrm(a24 - b42), nrm(a13 - b24) + nrm(a24 - b13),
         nrm(a13 - b31) + nrm(a24 - b24), nrm(a13 - b42) + nrm(a24 - b31)]
    iori, ss = -1, 1.0e-3 * chlref
    for q in range(4):
        if s[q] < ss:
            iori, ss = q, s[q]
    return iori


def orient_connections(blocks, chlref=1.0):
    """The orientation (ICON(14), ORIENT's turn, gluebm.f:8188) of every 1:1
    patch of the blocks (each with its nodes), from its corners and its
    partner's: the patch on block IBTYPE, face NFACE starting at (N1A,
    N2A).  Raises where no orientation matches."""
    for b in blocks:
        for pa in b.patches:
            if pa.ityp != grid.BC_CON:
                continue
            nb = blocks[pa.ibtype]
            part = [q for q in nb.patches if q.ityp == grid.BC_CON and q.iface == pa.nface
                    and q.r1a == pa.n1a and q.r2a == pa.n2a]
            if not part:
                raise ValueError(f"1:1 patch on face {pa.iface}: no partner on block {pa.ibtype} face {pa.nface}")
            q = part[0]
            xcol = patch_corners(b.nodes, pa.iface, (pa.r1a, pa.r1b), (pa.r2a, pa.r2b))
            xcog = patch_corners(nb.nodes, q.iface, (q.r1a, q.r1b), (q.r2a, q.r2b))
            iori = orient(xcol, xcog, chlref)
            if iori < 0:
                raise ValueError(f"1:1 patch on face {pa.iface}: the patch orientation cannot be solved")
            pa.iori = iori
    return blocks


def init_freestream(b: Block, fs, *, noise=1e-3, seed=0):
    """Uniform free stream plus seeded Gaussian noise on the density of the
    interior cells, held at constant pressure (T = p/(R rho))."""
    a = b.arrays
    a["TEMP"][:] = fs["t"]
    a["U"][:] = fs["u"]
    a["V"][:] = 0.0
    a["W"][:] = 0.0
    a["PDIFF"][:] = 0.0
    a["EPS2"][:] = 1.0
    a["VIST"][:] = 0.0
    if noise:
        rng = np.random.default_rng(seed)
        n = rng.standard_normal(b.interior_cells).reshape(b.kmax, b.jmax, b.imax)
        rho = fs["rho"] * (1.0 + noise * n)
        b.interior("TEMP")[:] = fs["p"] / (287.05287 * rho)
    return b


# ---- wall distance (DISTANCES gluebm.f:9136) ---------------------------------

def _kpass_centres(P):
    """AREVC1's cell centres (its last, k-direction pass: corners at the
    offsets 0, j, i+j, i, k, k+j, k+i+j, k+i, summed in that order) of the
    cells spanned by the node array P [k, j, i, 3]."""
    nk, nj, ni = P.shape[0] - 1, P.shape[1] - 1, P.shape[2] - 1

    def c(di, dj, dk):
        return P[dk:dk + nk, dj:dj + nj, di:di + ni]

    return 0.125 * (c(0, 0, 0) + c(0, 1, 0) + c(1, 1, 0) + c(1, 0, 0) + c(0, 0, 1) + c(0, 1, 1) + c(1, 1, 1)
                    + c(1, 0, 1))


def wall_points(nodes, patches):
    """PICK_XYZ gluebm.f:9452 for one block: the points halfway between the
    centre of the first interior cell and of the first ghost cell at every
    cell of its solid patches (ICON(1) 8..10), [n, 3], in patch order and,
    within a patch, the second in-face index outermost.  The centres are
    AREVC1's (the ghost cell's nodes reflected through the face, GRIDEX)."""
    X, Y, Z = nodes
    P = np.stack([X, Y, Z], axis=-1)
    out = []
    for pa in patches:
        if not 8 <= pa.ityp <= 10:
            continue
        d = (pa.iface - 1) % 3          # 0 = i, 1 = j, 2 = k
        ax = 2 - d                      # its axis of P
        n = P.shape[ax]
        if pa.iface <= 3:               # the reflected node plane, then planes 0 and 1
            pl = [2 * np.take(P, 0, axis=ax) - np.take(P, 1, axis=ax), np.take(P, 0, axis=ax),
                  np.take(P, 1, axis=ax)]
        else:
            pl = [np.take(P, n - 2, axis=ax), np.take(P, n - 1, axis=ax),
                  2 * np.take(P, n - 1, axis=ax) - np.take(P, n - 2, axis=ax)]
        slab = np.stack(pl, axis=ax)
        cen = _kpass_centres(slab)                   # two cells along the normal
        lo, hi = np.take(cen, 0, axis=ax), np.take(cen, 1, axis=ax)
        pt = 0.5 * (lo + hi)                         # XC(KMI) + XC(KMA): the lower cell first
        # pt is [second, first] in-face index for every face direction
        sub = pt[pa.r2a - 1:pa.r2b, pa.r1a - 1:pa.r1b]
        out.append(sub.reshape(-1, 3))
    return np.concatenate(out) if out else np.zeros((0, 3))


def wall_distance_points(blk: Block, pts, ncand: int = 8):
    """WALL_DIST gluebm.f:9533: DISTW of every storage cell of blk, the
    distance of its centre to the nearest wall point (squared distances
    (dx^2 + dy^2) + dz^2 compared, the root of the least; 1e4 without
    points, the root of DISTANCES' initial 1e8).  The ncand points nearest
    by a k-d tree are the candidates."""
    if not len(pts):
        return np.full(blk.ntot, 1.0e4)
    from scipy.spatial import cKDTree
    q = np.stack([blk.arrays["XC"], blk.arrays["YC"], blk.arrays["ZC"]], axis=1)
    k = min(ncand, len(pts))
    _, idx = cKDTree(pts).query(q, k=k, workers=-1)
    idx = idx.reshape(len(q), k)
    best = np.full(len(q), 1.0e8)
    for j in range(k):
        p = pts[idx[:, j]]
        dx, dy, dz = q[:, 0] - p[:, 0], q[:, 1] - p[:, 1], q[:, 2] - p[:, 2]
        r = dx * dx + dy * dy + dz * dz
        best = np.where(r < best, r, best)
    return np.sqrt(best)


def lump_wall_distance(fine: Block, coarse: Block):
    """LUMP_DIST gluebm.f:9562: the coarse interior cells' DISTW, the mean
    of their eight children in LUMPVS's order (in place; the coarse ghost
    cells keep theirs)."""
    f = fine.arrays["DISTW"].reshape(fine.kmax + 4, fine.jmax + 4, fine.imax + 4)
    c = coarse.arrays["DISTW"].reshape(coarse.kmax + 4, coarse.jmax + 4, coarse.imax + 4)
    ci, cj, ck = coarse.imax, coarse.jmax, coarse.kmax

    def child(di, dj, dk):
        return f[2 + dk:2 + dk + 2 * ck:2, 2 + dj:2 + dj + 2 * cj:2, 2 + di:2 + di + 2 * ci:2]

    ra = child(0, 0, 0)
    for o in ((0, 1, 0), (0, 0, 1), (0, 1, 1), (1, 0, 0), (1, 1, 0), (1, 0, 1), (1, 1, 1)):
        ra = ra + child(*o)
    c[2:-2, 2:-2, 2:-2] = 0.125 * ra


def sst_freestream(fs, tu=1.0e-3, mut_ratio=0.1):
    """Free-stream rho*k and rho*omega from the turbulence intensity and
    mu_t/mu (main.f:3770-3790, IDIS=2): rho*k = 1.5 rho (Tu U)^2,
    rho*omega = rho (rho*k) / mu_t."""
    rk = 1.5 * fs["rho"] * (tu * fs["u"]) ** 2
    mut = mut_ratio * fs["mu"]
    return rk, fs["rho"] * rk / mut


def bump_case(ni=65, nj=33, nk=33, *, h1=1e-3, amp=0.1, mach=0.5, reynolds=1e4,
              zlen=0.5, noise=1e-3, seed=0, cfl=2.0, inter=3, span_amp=0.0,
              turbulence=None, tu=1.0e-3, mut_ratio=0.1):
    """The single-block bump channel (node counts ni x nj x nk); laminar, or
    k-omega SST with turbulence="sst" (free-stream Tu and mu_t/mu)."""
    fc = FlowConditions(mach=mach, reynolds=reynolds)
    fs = fc.freestream()
    X, Y, Z = grid.bump_nodes(ni, nj, nk, h1=h1, amp=amp, zlen=zlen, span_amp=span_amp)
    imax, jmax, kmax = ni - 1, nj - 1, nk - 1
    blk = new_block(X, Y, Z, channel_patches(imax, jmax, kmax, fs))
    init_freestream(blk, fs, noise=noise, seed=seed)
    prm = make_params(fc, blk.dims, cfl=cfl, inter=inter)
    if turbulence == "sst":
        setup_sst(blk, prm, fs, tu=tu, mut_ratio=mut_ratio)
    return blk, prm, fs


def setup_sst(blk: Block, prm: FFParams, fs, tu=1.0e-3, mut_ratio=0.1, walls=None, fine: Block = None,
              distw=True):
    """Switch a case to k-omega SST: ITURB=6, the free-stream limits RKLIM /
    EPSLIM, inlet BOUNRK/BOUNEP, DISTW, and rho*k, rho*omega, mu_t of the
    free stream in every cell.  DISTW: the distance to the wall points
    `walls` (default: blk's own solid patches, from its nodes); a coarse
    level passes its finer level as `fine`, whose DISTW its interior cells
    average (LUMP_DIST).  distw=False leaves it to the device
    (ff_wall_distance)."""
    rk, re = sst_freestream(fs, tu, mut_ratio)
    prm.iturb = 6
    prm.rklim, prm.epslim = rk, re
    for pa in blk.patches:
        pa.bounrk, pa.bounep = rk, re
    if distw:
        if walls is None:
            walls = wall_points(blk.nodes, blk.patches)
        blk.arrays["DISTW"][:] = wall_distance_points(blk, walls)
        if fine is not None:
            lump_wall_distance(fine, blk)
    blk.arrays["RK"][:] = rk
    blk.arrays["REPS"][:] = re
    blk.arrays["EPS2"][:] = 1.0 + mut_ratio
    blk.arrays["VIST"][:] = mut_ratio * fs["mu"]
    blk.arrays["RKOLD"][:] = rk
    blk.arrays["EPSOLD"][:] = re
    return blk


def bump_case_mg(ni=65, nj=33, nk=33, nlev=3, *, h1=1e-3, amp=0.1, mach=0.5, reynolds=1e4,
                 zlen=0.5, noise=1e-3, seed=0, cfl=2.0, cfll=2.0, inter=3, span_amp=0.0,
                 lusgs_fp32=False, coarse_fp32=False, coarse_res_fp32=False, turbulence=None, tu=1.0e-3,
                 mut_ratio=0.1):
    """The bump channel with nlev multigrid levels (finest first); coarse
    metrics are lumped from the fine cells, patch ranges follow each level.
    lusgs_fp32 runs the fine level's implicit operator in FP32, coarse_fp32
    the coarse levels' (their correction reaches the fine level through
    INTERP), coarse_res_fp32 the coarse levels' face fluxes; the fine
    level's residual, every update and the norms stay FP64."""
    fc = FlowConditions(mach=mach, reynolds=reynolds)
    fs = fc.freestream()
    X, Y, Z = grid.bump_nodes(ni, nj, nk, h1=h1, amp=amp, zlen=zlen, span_amp=span_amp)
    levels = []
    for lev, m in enumerate(grid.mg_metrics(X, Y, Z, nlev)):
        blk = block_from_metrics(m, channel_patches(m.imax, m.jmax, m.kmax, fs), nodes=(X, Y, Z) if lev == 0 else None)
        init_freestream(blk, fs, noise=noise if lev == 0 else 0.0, seed=seed)
        levels.append(blk)
    prm = make_params(fc, levels[0].dims, cfl=cfl, cfll=cfll, inter=inter)
    if turbulence == "sst":
        walls = wall_points(levels[0].nodes, levels[0].patches)
        for lev, blk in enumerate(levels):
            setup_sst(blk, prm if lev == 0 else FFParams.from_buffer_copy(prm), fs, tu=tu,
                      mut_ratio=mut_ratio, walls=walls, fine=levels[lev - 1] if lev else None)
    prms = [level_params(prm, lev + 1) for lev in range(nlev)]
    prms[0].lusgs_fp32 = int(lusgs_fp32)
    for q in prms[1:]:
        q.lusgs_fp32 = int(coarse_fp32)
        q.res_fp32 = int(coarse_res_fp32)
    return levels, prms, fs


# ---- multi-block periodic box (1:1 patched blocks) -----------------------

_OPP = {1: 4, 2: 5, 3: 6, 4: 1, 5: 2, 6: 3}


def _face_ranges(iface, imax, jmax, kmax):
    d = (iface - 1) % 3
    if d == 0:
        return (1, jmax), (1, kmax)
    if d == 1:
        return (1, imax), (1, kmax)
    return (1, imax), (1, jmax)


def box_block_sizes(nb=(4, 3, 2), seed=2, target=6.0e6, tol=0.10, nodes=tuple(range(17, 98, 4))):
    """Cells per block along each direction of the Cartesian block
    arrangement: node counts drawn with the seed from {17, 21, ..., 97} (one
    more than a multiple of 4, so every block has three multigrid levels),
    redrawn until the total is within tol of target cells.  Block (a, b, c)
    has (ni[a], nj[b], nk[c]) cells, so every interface is 1:1."""
    rng = np.random.default_rng(seed)
    nodes = np.asarray(nodes)
    for _ in range(100000):
        s = tuple([int(v) - 1 for v in rng.choice(nodes, size=n)] for n in nb)
        cells = sum(s[0]) * sum(s[1]) * sum(s[2])
        if abs(cells - target) <= tol * target:
            return s
    raise RuntimeError("no block split within the target size")


def periodic_box_case(nb=(4, 3, 2), sizes=None, *, seed=2, mach=0.3, target=None,
                      amp=1e-2, cfl=2.0, inter=3, lusgs_fp32=False, wave=(1, 1, 1)):
    """The unit box split into nb[0] x nb[1] x nb[2] blocks with 1:1 patches on
    every interface, periodic in all three directions (the outer faces are
    1:1 patched to the opposite blocks).  Inviscid (viscous face fluxes off,
    IDI1..3 = 0) uniform flow at the given Mach number along the diagonal,
    with an entropy wave rho = rho0 (1 + amp sin(2 pi k.x + phi)) at constant
    pressure; phi comes from the seed.  Returns blocks, params, free stream."""
    if sizes is None:
        # 6M cells for the 24-block arrangement, proportionally fewer otherwise
        tgt = target if target is not None else 6.0e6 * nb[0] * nb[1] * nb[2] / 24
        sizes = box_block_sizes(nb, seed, target=tgt)
    ni, nj, nk = sizes
    fc = FlowConditions(mach=mach, reynolds=0.0)
    fs = fc.freestream()
    phi = 2 * math.pi * np.random.default_rng(seed + 1000).random()
    cut = [np.concatenate([[0], np.cumsum(n)]) for n in (ni, nj, nk)]
    tot = [c[-1] for c in cut]
    ids = {}
    for c in range(len(nk)):
        for b in range(len(nj)):
            for a in range(len(ni)):
                ids[a, b, c] = len(ids)
    blocks, prms = [], []
    u = fs["u"] / math.sqrt(3.0)
    for (a, b, c), bid in ids.items():
        x = cut[0][a:a + 2]; y = cut[1][b:b + 2]; z = cut[2][c:c + 2]
        X, Y, Z = grid.box_nodes(np.arange(x[0], x[1] + 1) / tot[0],
                                 np.arange(y[0], y[1] + 1) / tot[1],
                                 np.arange(z[0], z[1] + 1) / tot[2])
        imax, jmax, kmax = ni[a], nj[b], nk[c]
        pats = []
        for iface in range(1, 7):
            d = (iface - 1) % 3
            step = -1 if iface <= 3 else 1
            nbr = [a, b, c]
            nbr[d] = (nbr[d] + step) % len(sizes[d])
            r1, r2 = _face_ranges(iface, imax, jmax, kmax)
            pa = _patch(grid.BC_CON, iface, r1, r2, ibtype=ids[tuple(nbr)])
            pa.nface = _OPP[iface]
            pa.n1a = pa.n2a = 1
            pats.append(pa)
        blk = new_block(X, Y, Z, pats)
        ar = blk.arrays
        ar["TEMP"][:] = fs["t"]
        ar["U"][:] = u; ar["V"][:] = u; ar["W"][:] = u
        ar["PDIFF"][:] = 0.0
        ar["EPS2"][:] = 1.0
        ar["VIST"][:] = 0.0
        xc, yc, zc = (blk.interior(n) for n in ("XC", "YC", "ZC"))
        arg = 2 * math.pi * (wave[0] * xc + wave[1] * yc + wave[2] * zc) + phi
        rho = fs["rho"] * (1.0 + amp * np.sin(arg))
        blk.interior("TEMP")[:] = fs["p"] / (fc.rgas * rho)
        prm = make_params(fc, blk.dims, cfl=cfl, inter=inter, fullns=False, lusgs_fp32=lusgs_fp32)
        prm.idi1 = prm.idi2 = prm.idi3 = 0
        blocks.append(blk)
        prms.append(prm)
    orient_connections(blocks)
    return blocks, prms, fs


# ---- multi-block bump with multigrid levels (the large combined case) -------

def bump_block_cuts(cells, nb, seed, quantum=4, spread=0.1):
    """Uneven cut positions of each direction: nb[d] blocks whose sizes are
    multiples of `quantum` cells (so every block has its multigrid levels),
    each within +-spread of the even split, drawn with the seed."""
    rng = np.random.default_rng(seed)
    cuts = []
    for n, m in zip(cells, nb):
        base = n / m
        pos = [0]
        for q in range(1, m):
            jit = int(round(rng.uniform(-spread, spread) * base / quantum)) * quantum
            pos.append(int(round(q * base / quantum)) * quantum + jit)
        pos.append(n)
        cuts.append(pos)
    return cuts


def channel_wall_points(X, Y, Z):
    """The wall points of the whole channel's lower and upper walls: those
    of the solid j faces of all its blocks (the nearest point does not
    depend on their order)."""
    kmax, imax = X.shape[0] - 1, X.shape[2] - 1
    pats = [_patch(grid.BC_SOL, 2, (1, imax), (1, kmax)), _patch(grid.BC_SOL, 5, (1, imax), (1, kmax))]
    return wall_points((X, Y, Z), pats)


def bump_multiblock_blocks(cells=(512, 256, 128), nb=(2, 2, 2), nlev=3, *, seed=5, h1=2e-6, amp=0.1,
                           span_amp=0.5, zlen=1.0, mach=0.7, reynolds=5e6, noise=1e-3, cfl=1.0, cfll=1.0,
                           inter=3, turbulence="sst", tu=1.0e-3, mut_ratio=0.1, lusgs_fp32=True,
                           coarse_fp32=True, coarse_res_fp32=False, device_setup=False):
    """The bump channel split into nb[0] x nb[1] x nb[2] blocks of uneven
    sizes (cut positions from the seed), 1:1 patched on every interior cut,
    periodic in z through 1:1 patches (the spanwise amplitude
    a(z) = amp (1 + span_amp sin 2 pi z) is periodic on [0, zlen = 1]),
    INL / OUT / SOL on the outer i and j faces.  Yields, block by block
    (i fastest), (levels, prms) with nlev multigrid levels each; a 1:1
    patch's IBTYPE is the source block's index.  Block metrics take mirror
    ghost nodes at the cuts as well (the interface faces themselves are
    exact); the wall distance is to the walls of the whole channel.  Also
    yields the free stream first: the first item is ("fs", fs).  With
    device_setup the metric arrays and DISTW are left at zero for
    ff_block_metrics_levels / ff_wall_distance: the second item is then
    ("wall", points) (the channel's wall points, [n, 3]), and each level-1
    block carries its nodes."""
    fc = FlowConditions(mach=mach, reynolds=reynolds)
    fs = fc.freestream()
    yield "fs", fs
    NI, NJ, NK = cells
    X, Y, Z = grid.bump_nodes(NI + 1, NJ + 1, NK + 1, h1=h1, amp=amp, zlen=zlen, span_amp=span_amp)
    wall = channel_wall_points(X, Y, Z)
    if device_setup:
        yield "wall", wall
    cut = bump_block_cuts(cells, nb, seed)
    ids = {}
    for c in range(nb[2]):
        for b in range(nb[1]):
            for a in range(nb[0]):
                ids[a, b, c] = len(ids)
    inl = dict(bounr=fs["rho"], bounu=fs["u"], bounv=0.0, bounw=0.0, bount=fs["t"], bounp=fs["p"], bounpd=0.0)
    for (a, b, c), bid in ids.items():
        i0, i1 = cut[0][a], cut[0][a + 1]
        j0, j1 = cut[1][b], cut[1][b + 1]
        k0, k1 = cut[2][c], cut[2][c + 1]
        Xb, Yb, Zb = (np.ascontiguousarray(A[k0:k1 + 1, j0:j1 + 1, i0:i1 + 1]) for A in (X, Y, Z))
        levels = []
        if device_setup:   # dimensions only; the device fills the metrics
            mets = [grid.Metrics((i1 - i0) >> lev, (j1 - j0) >> lev, (k1 - k0) >> lev) for lev in range(nlev)]
            for m in mets:
                m.arrays = {n: np.zeros(m.ntot) for n in grid.METRIC_NAMES}
        else:
            mets = grid.mg_metrics(Xb, Yb, Zb, nlev)
        for lev, m in enumerate(mets):
            pats = []
            for iface in range(1, 7):
                d = (iface - 1) % 3
                r1, r2 = _face_ranges(iface, m.imax, m.jmax, m.kmax)
                pos = (a, b, c)[d]
                last = pos == nb[d] - 1
                outer = (iface <= 3 and pos == 0) or (iface > 3 and last)
                if outer and d == 0:
                    pats.append(_patch(grid.BC_INL if iface == 1 else grid.BC_OUT, iface, r1, r2,
                                       ibtype=4 if iface == 1 else 3, **inl))
                elif outer and d == 1:
                    pats.append(_patch(grid.BC_SOL, iface, r1, r2))
                else:   # interior cut, or the periodic z faces
                    nbr = [a, b, c]
                    nbr[d] = (nbr[d] + (-1 if iface <= 3 else 1)) % nb[d]
                    pa = _patch(grid.BC_CON, iface, r1, r2, ibtype=ids[tuple(nbr)])
                    pa.nface = _OPP[iface]
                    pa.n1a = pa.n2a = 1
                    pats.append(pa)
            blk = block_from_metrics(m, pats, nodes=(Xb, Yb, Zb) if lev == 0 else None)
            init_freestream(blk, fs, noise=noise if lev == 0 else 0.0, seed=seed + 100 * bid)
            levels.append(blk)
        prm = make_params(fc, levels[0].dims, cfl=cfl, cfll=cfll, inter=inter)
        if turbulence == "sst":
            for lev, blk in enumerate(levels):
                setup_sst(blk, prm if lev == 0 else FFParams.from_buffer_copy(prm), fs, tu=tu,
                          mut_ratio=mut_ratio, walls=wall, fine=levels[lev - 1] if lev else None,
                          distw=not device_setup)
        prms = [level_params(prm, lev + 1) for lev in range(nlev)]
        prms[0].lusgs_fp32 = int(lusgs_fp32)
        for q in prms[1:]:
            q.lusgs_fp32 = int(coarse_fp32)
            q.res_fp32 = int(coarse_res_fp32)
        yield levels, prms


def bump_multiblock_case(*args, **kw):
    """All blocks of bump_multiblock_blocks at once: (block_levels,
    block_prms, fs), and the wall points last with device_setup."""
    it = bump_multiblock_blocks(*args, **kw)
    _, fs = next(it)
    tri = next(it)[1] if kw.get("device_setup") else None
    bl, bp = [], []
    for levels, prms in it:
        bl.append(levels)
        bp.append(prms)
    orient_connections([lv[0] for lv in bl])
    return (bl, bp, fs, tri) if tri is not None else (bl, bp, fs)


# ---- patches from / to FINFLO's BC file (READBC gluebm.f:2553) -------------

def patches_from_bc(bc_patches, nblocks, fs, rk=0.0, reps=0.0):
    """The library's patch tables (one FFPatch list per block, file order)
    from the patches fileio.read_bc returns.  Inlet/outlet boundary values
    are the free stream's, uniform over the patch (the boundary-value files
    are not read); a connection's IBTYPE is its source block's 0-based index,
    NFACE its face and N1A/N2A the start of the matching range.  A
    connection's orientation ICON(14) comes from the grid: orient_connections
    on the blocks built with these tables."""
    out = [[] for _ in range(nblocks)]
    inl = dict(bounr=fs["rho"], bounu=fs["u"], bounv=0.0, bounw=0.0, bount=fs["t"], bounp=fs["p"], bounpd=0.0,
               bounrk=rk, bounep=reps)
    for p in bc_patches:
        if p.ityp == grid.BC_CON:
            pa = _patch(grid.BC_CON, p.iface, (p.r1a, p.r1b), (p.r2a, p.r2b), ibtype=p.nblock - 1)
            pa.nface, pa.n1a, pa.n2a = p.nface, p.n1a, p.n2a
        elif p.ityp in (grid.BC_INL, grid.BC_OUT):
            pa = _patch(p.ityp, p.iface, (p.r1a, p.r1b), (p.r2a, p.r2b), ibtype=p.itype, **inl)
        elif p.ityp in (grid.BC_SOL, grid.BC_MIR):
            pa = _patch(p.ityp, p.iface, (p.r1a, p.r1b), (p.r2a, p.r2b), iheat=p.iheat if p.ityp == grid.BC_SOL else 0)
        else:
            raise ValueError(f"BC type {p.kind} is not on this path")
        out[p.block - 1].append(pa)
    return out


def bc_from_patches(block_patches, periodic_faces=()):
    """The BC-file patches (fileio.BcPatch) of the library's patch tables:
    the inverse of patches_from_bc.  A connection through a face listed in
    periodic_faces is written as PER."""
    from . import fileio
    names = {grid.BC_INL: "INL", grid.BC_OUT: "OUT", grid.BC_SOL: "SOL", grid.BC_MIR: "MIR", grid.BC_CON: "CON"}
    out = []
    for ib, pats in enumerate(block_patches, start=1):
        seen = {}
        for pa in pats:
            seen[pa.iface] = seen.get(pa.iface, 0) + 1
            kind = names[pa.ityp]
            if kind == "CON" and pa.iface in periodic_faces:
                kind = "PER"
            p = fileio.BcPatch(kind, ib, pa.iface, seen[pa.iface])
            p.r1a, p.r1b, p.r2a, p.r2b = pa.r1a, pa.r1b, pa.r2a, pa.r2b
            if pa.ityp == grid.BC_CON:
                p.nblock, p.nface = pa.ibtype + 1, pa.nface
            elif pa.ityp in (grid.BC_INL, grid.BC_OUT):
                p.itype = pa.ibtype
                p.bfile = "INLET.DAT" if pa.ityp == grid.BC_INL else "OUTLET.DAT"
            elif pa.ityp == grid.BC_SOL:
                p.iheat = pa.iheat
                p.rcon = [0.0] * 13 + [1.0]
            out.append(p)
    # a connection names its partner by the partner's position on its face
    for p in out:
        if p.kind in ("CON", "PER"):
            pa = block_patches[p.block - 1][[q for q in out if q.block == p.block].index(p)]
            cands = [q for q in out if q.block == p.nblock and q.iface == p.nface and q.kind in ("CON", "PER")]
            match = [q for q in cands if q.r1a <= pa.n1a <= q.r1b and q.r2a <= pa.n2a <= q.r2b]
            if not match:
                raise ValueError(f"block {p.block} face {p.iface}: no partner patch")
            p.npatch = match[0].local
    return out
