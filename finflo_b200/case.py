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
                ("bounpd", ctypes.c_double)]


class FFParams(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in (
        "gamma", "rgas", "pr", "prt", "visu0", "expsu", "tsu0", "e0ref", "t0ref",
        "frsden", "frspre", "frsvel", "frsvis", "frstem", "cfl", "cfll", "theta",
        "cdiff", "pvisc", "tlolim", "tuplim", "cmgk", "cmgeps")] + [
        (n, ctypes.c_int) for n in (
            "interi", "interj", "interk", "entropy_fix", "iturb", "fullns",
            "idi1", "idi2", "idi3", "coarse_inter", "lusgs_fp32", "pad0")]


# enum ff_slot (include/finflo_types.h), in order
SLOTS = ["RO", "RM", "RN", "RW", "E", "P", "PDIFF", "U", "V", "W", "C",
         "TEMP", "VIS", "CH", "CP", "DRDP", "DRDH", "EPS2", "VIST",
         "DRO", "DM", "DN", "DW", "DE", "DTL",
         "TOLD", "UOLD", "VOLD", "WOLD", "POLD",
         "A1", "A1XA", "A1YA", "A1ZA", "A2", "A2XA", "A2YA", "A2ZA",
         "A3", "A3XA", "A3YA", "A3ZA", "VOL", "XC", "YC", "ZC", "D1", "D2", "D3",
         "W12", "W13", "W23", "S11", "S12", "S13", "S22", "S23", "S33",
         "DTDX", "DTDY", "DTDZ", "OHMI", "STRAIN",
         "F1R", "F1RM", "F1RN", "F1RW", "F1E",
         "ROP2H", "RMP2H", "RNP2H", "RWP2H", "EP2H"]
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


def make_params(fc: FlowConditions, dims, *, cfl=2.0, cfll=2.0, inter=3,
                fullns=True, iturb=0, entropy_fix=False, lusgs_fp32=False) -> FFParams:
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
    p.interi = p.interj = p.interk = inter
    p.entropy_fix = int(entropy_fix)
    p.iturb = iturb
    p.fullns = int(fullns)
    imax, jmax, kmax = dims
    # IDI1..3 default to the node counts (main.f:5657-5659): viscous everywhere
    p.idi1, p.idi2, p.idi3 = imax + 1, jmax + 1, kmax + 1
    p.coarse_inter = 55
    p.lusgs_fp32 = int(lusgs_fp32)
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


def bump_case(ni=65, nj=33, nk=33, *, h1=1e-3, amp=0.1, mach=0.5, reynolds=1e4,
              zlen=0.5, noise=1e-3, seed=0, cfl=2.0, inter=3, span_amp=0.0):
    """The single-block laminar bump channel (node counts ni x nj x nk)."""
    fc = FlowConditions(mach=mach, reynolds=reynolds)
    fs = fc.freestream()
    X, Y, Z = grid.bump_nodes(ni, nj, nk, h1=h1, amp=amp, zlen=zlen, span_amp=span_amp)
    imax, jmax, kmax = ni - 1, nj - 1, nk - 1
    blk = new_block(X, Y, Z, channel_patches(imax, jmax, kmax, fs))
    init_freestream(blk, fs, noise=noise, seed=seed)
    prm = make_params(fc, blk.dims, cfl=cfl, inter=inter)
    return blk, prm, fs
