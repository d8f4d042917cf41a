"""Learned warm start: a small network predicts the flow field of a bump
channel from its parameters (free-stream Mach number, bump amplitude); the
solver then iterates from that prediction instead of from the free stream,
to the same residual tolerance, and stays the judge of the prediction.

Network (BF16 weights, FP32 accumulation, every product on the tensor cores
through libfinflo_nn.so):

* encoder: a 4-layer MLP on the normalised parameters (2 -> 64 -> 128 ->
  256 -> 512), SiLU between layers; the 512 outputs are a 4x2x2 grid of
  32-channel root voxels;
* decoder: four levels of a 3-D transposed convolution with kernel 2 and
  stride 2 (each voxel -> its 2x2x2 children, 32 -> 8 x 32 channels, SiLU)
  followed by a 1x1x1 convolution (32 -> 32, SiLU), then a 1x1x1 output
  convolution to the 5 conservative variables of each of the 64x32x32
  cells.  Voxels are kept in octree order (child index = 8 x parent +
  octant), so each transposed convolution is one GEMM whose output rows are
  already the next level's voxels.

Targets are the conservative variables (RO, RM, RN, RW, E) of converged
solver runs, scaled by each case's free-stream values, minus their mean over
the training set per cell, divided by one spread per variable (the
spanwise momentum, numerical noise in these spanwise-uniform cases, shares
the normal momentum's spread so that it does not weigh in the loss).
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field

import numpy as np

CH = 32                # decoder channels
OUT_PAD = 16           # output channels padded to the GEMM's N step
IN_PAD = 16            # parameters padded to the GEMM's K step


@dataclass(frozen=True)
class Spec:
    """A family of cases the network learns: the solver case built from the
    parameters, the decoder's grid (root voxels refined `levels` times) and
    the predicted variables (5 conservative, or 7 with k and omega)."""
    name: str
    root: tuple = (4, 2, 2)
    levels: int = 4
    nvar: int = 5
    params: tuple = ("mach", "amp")
    ranges: tuple = ((0.3, 0.8), (0.05, 0.15))
    nodes: tuple = (65, 33, 33)
    nlev: int = 1                       # solver multigrid levels
    reynolds: float = 1e4
    h1: float = 1e-3
    noise: float = 1e-3
    amp: float = 0.1                    # bump amplitude when it is not a parameter
    inter: int = 3
    cfl: float = 2.0
    turbulence: str = None
    span_amp: float = 0.0               # spanwise bump variation a(z) = amp (1 + span_amp sin 2 pi z)
    zlen: float = 0.5                   # spanwise extent

    @property
    def grid(self):
        return tuple(r << self.levels for r in self.root)

    @property
    def ncell(self):
        g = self.grid
        return g[0] * g[1] * g[2]

    @property
    def enc(self):
        return [IN_PAD, 64, 128, 256, CH * self.root[0] * self.root[1] * self.root[2]]


# the config-4 family: laminar bump channel 64x32x32, Mach and bump amplitude
BUMP = Spec("laminar bump channel 64x32x32 cells, Re 1e4, Mach U[0.3,0.8], amplitude U[0.05,0.15]")
# the SST bump channel of the V-cycle workload (128x64x64, first cell 2e-6,
# Re 1e6, 3 levels, INTER=1, CFL 1) over a subsonic Mach sweep around its
# M = 0.6; predicts k and omega too.  (From M ~ 0.69 on, a supersonic pocket
# forms over the bump; predicted starts there diverged and the plain solver
# took over, so the family stops at 0.65.)
SST = Spec("k-omega SST bump channel 128x64x64 cells, Re 1e6, first cell 2e-6, 3-level V-cycle, Mach U[0.5,0.65]",
           root=(4, 2, 2), levels=5, nvar=7, params=("mach",), ranges=((0.5, 0.65),), nodes=(129, 65, 65), nlev=3,
           reynolds=1e6, h1=2e-6, noise=1e-3, inter=1, cfl=1.0, turbulence="sst")

# the config-5 geometry (the spanwise-varying bump, amplitude
# 0.1 (1 + 0.5 sin 2 pi z) on z in [0, 1], k-omega SST, Re 5e6, first cell
# 2e-6, 3-level V-cycles, INTER=1, CFL 1) as one 128x64x64-cell block with
# slip spanwise faces, over a Mach sweep below the transonic pocket; the
# family the network is retrained on for config 5 (32 solutions), at the
# single-block size the solves fit in (the 16.8 M-cell eight-block case
# itself costs ~2 min of GPU per solution)
SST5 = Spec("config-5 geometry: k-omega SST spanwise-varying bump 128x64x64 cells, amplitude 0.1(1+0.5 sin 2 pi z), "
            "z in [0,1], Re 5e6, first cell 2e-6, 3-level V-cycle, Mach U[0.5,0.65]",
            root=(4, 2, 2), levels=5, nvar=7, params=("mach",), ranges=((0.5, 0.65),), nodes=(129, 65, 65), nlev=3,
            reynolds=5e6, h1=2e-6, noise=1e-3, inter=1, cfl=1.0, turbulence="sst", span_amp=0.5, zlen=1.0)

# the config-4 family's sizes, kept as module constants
ROOT, LEVELS, NVAR = BUMP.root, BUMP.levels, BUMP.nvar
ENC = BUMP.enc
GRID = BUMP.grid   # cells: 64, 32, 32


def octree_order(root=ROOT, levels=LEVELS):
    """Interior cell index (i fastest, [k][j][i]) of each finest-level voxel
    in decoder order.  Root r = (rk * Rj + rj) * Ri + ri; a child's index is
    8 x parent + (di + 2 dj + 4 dk)."""
    ri, rj, rk = np.meshgrid(np.arange(root[0]), np.arange(root[1]), np.arange(root[2]), indexing="ij")
    # voxel coordinates at level 0, in root order
    order = np.argsort((rk * root[1] + rj) * root[0] + ri, axis=None, kind="stable")
    I, J, K = ri.ravel()[order], rj.ravel()[order], rk.ravel()[order]
    for _ in range(levels):
        c = np.arange(8)
        di, dj, dk = c & 1, (c >> 1) & 1, (c >> 2) & 1
        I = (2 * I[:, None] + di[None, :]).ravel()
        J = (2 * J[:, None] + dj[None, :]).ravel()
        K = (2 * K[:, None] + dk[None, :]).ravel()
    ni, nj = root[0] << levels, root[1] << levels
    return (K * nj + J) * ni + I


QVARS = ("RO", "RM", "RN", "RW", "E", "RK", "REPS")


def conservative(blk, nvar=5):
    """Interior (RO, RM, RN, RW, E[, RK, REPS]) of a block as [cells, nvar],
    i fastest."""
    return np.stack([blk.interior(n).ravel() for n in QVARS[:nvar]], axis=1)


def freestream_scales(fs, gamma=1.4, rgas=287.05287):
    """Per-variable scales of a case (fs: the free-stream dict of
    FlowConditions): rho, rho U, rho U, rho U, E."""
    ru = fs["rho"] * fs["u"]
    e = fs["rho"] * (rgas * fs["t"] / (gamma - 1.0) + 0.5 * fs["u"] ** 2)
    return np.array([fs["rho"], ru, ru, ru, e])


def state_from_conservative(q, fs, gamma=1.4, rgas=287.05287):
    """Solver state (TEMP, U, V, W, PDIFF) of conservative values q [cells, 5]
    for a perfect gas (PERFGA: e = R T / (gamma - 1), p = rho R T), with the
    density and temperature kept above a fraction of the free stream's;
    PDIFF is the pressure minus the free stream's (FRSPRE).  With q
    [cells, 7] (k and omega in columns 5, 6: rho k, rho omega) the internal
    energy excludes k, as CONSVA's E includes it, and RK, REPS are added."""
    ro = np.maximum(q[:, 0], 0.2 * fs["rho"])
    u, v, w = q[:, 1] / ro, q[:, 2] / ro, q[:, 3] / ro
    e = q[:, 4] / ro - 0.5 * (u * u + v * v + w * w)
    if q.shape[1] >= 7:
        e = e - q[:, 5] / ro
    T = np.maximum(e * (gamma - 1.0) / rgas, 0.2 * fs["t"])
    p = ro * rgas * T
    st = {"TEMP": T, "U": u, "V": v, "W": w, "PDIFF": p - fs["p"]}
    if q.shape[1] >= 7:
        st["RK"], st["REPS"] = q[:, 5], q[:, 6]
    return st


def normalise_params(*cols, spec=BUMP):
    """[n, IN_PAD] float32: each parameter column mapped from its range to
    [-1, 1] (normalise_params(mach, amp) for the config-4 family)."""
    n = len(cols[0])
    x = np.zeros((n, IN_PAD), dtype=np.float32)
    for c, (col, (lo, hi)) in enumerate(zip(cols, spec.ranges)):
        x[:, c] = 2.0 * (np.asarray(col) - lo) / (hi - lo) - 1.0
    return x


def _r16(n):
    return (n + 15) // 16 * 16


@dataclass
class Layer:
    name: str
    n: int            # outputs
    k: int            # inputs
    act: int          # 1: SiLU after the layer
    off: int = 0      # weight offset in the flat parameter buffer
    boff: int = 0     # bias offset


def layers(spec=BUMP):
    enc = spec.enc
    L = [Layer(f"enc{i + 1}", enc[i + 1], enc[i], 1 if i < 3 else 0) for i in range(4)]
    for lv in range(spec.levels):
        L.append(Layer(f"up{lv + 1}", 8 * CH, CH, 1))
        L.append(Layer(f"mix{lv + 1}", CH, CH, 1))
    L.append(Layer("out", OUT_PAD, CH, 0))
    off = 0
    for l in L:
        l.off = off
        off += l.n * l.k
    for l in L:
        l.boff = off
        off += l.n
    return L, off


class WarmStartNet:
    """Parameters, activations and the training step of the network.  torch
    holds the memory; every GEMM, activation gradient, reduction and the
    Adam update run in libfinflo_nn.so."""

    def __init__(self, device="cuda", seed=0, spec=BUMP):
        import torch
        from . import nn
        self.torch, self.nn = torch, nn
        self.spec = spec
        self.dev = torch.device(device)
        self.L, self.nparam = layers(spec)
        g = torch.Generator().manual_seed(seed)
        w = torch.zeros(self.nparam)
        for l in self.L:   # Kaiming-uniform weights for SiLU layers, zero biases
            bound = math.sqrt(6.0 / l.k) if l.act else math.sqrt(3.0 / l.k)
            if l.name == "enc1":
                bound = math.sqrt(6.0 / len(spec.params))   # the real inputs; the rest is padding
            w[l.off:l.off + l.n * l.k] = (torch.rand(l.n * l.k, generator=g) * 2 - 1) * bound
        self.w = w.to(self.dev)
        self.g = torch.zeros_like(self.w)
        self.m = torch.zeros_like(self.w)
        self.v = torch.zeros_like(self.w)
        self.w16 = torch.empty(self.nparam, dtype=torch.bfloat16, device=self.dev)
        self.w16t = torch.empty(self.nparam, dtype=torch.bfloat16, device=self.dev)
        self.step_n = 0
        self._sync_bf16()
        self.B = 0

    # -- parameter views ----------------------------------------------------
    def W(self, l):
        return self.w16[l.off:l.off + l.n * l.k].view(l.n, l.k)

    def WT(self, l):
        return self.w16t[l.off:l.off + l.n * l.k].view(l.k, l.n)

    def bias(self, l):
        return self.w[l.boff:l.boff + l.n]

    def gW(self, l):
        return self.g[l.off:l.off + l.n * l.k].view(l.n, l.k)

    def gb(self, l):
        return self.g[l.boff:l.boff + l.n]

    def _sync_bf16(self):
        nn = self.nn
        nn.to_bf16(self.w, self.w16)
        for l in self.L:
            nn.transpose(self.W(l), self.WT(l))

    # -- buffers ----------------------------------------------------------------
    def _alloc(self, B):
        if B == self.B:
            return
        torch = self.torch
        f32, b16, d = torch.float32, torch.bfloat16, self.dev
        self.B = B
        self.x0 = torch.zeros(B, IN_PAD, dtype=b16, device=d)
        self.z, self.h = {}, {"enc0": self.x0}
        for l in self.L[:4]:
            self.z[l.name] = torch.empty(B, l.n, dtype=f32, device=d)
            self.h[l.name] = torch.empty(B, l.n, dtype=b16, device=d)
        root = self.spec.root
        V = B * root[0] * root[1] * root[2]
        self.rows = {}
        prev = self.h["enc4"].view(V, CH)
        self.inp = {}
        for lv in range(self.spec.levels):
            up, mix = f"up{lv + 1}", f"mix{lv + 1}"
            self.inp[up] = prev
            self.z[up] = torch.empty(V, 8 * CH, dtype=f32, device=d)
            self.h[up] = torch.empty(V, 8 * CH, dtype=b16, device=d)
            self.rows[up] = V
            V *= 8
            self.inp[mix] = self.h[up].view(V, CH)
            self.z[mix] = torch.empty(V, CH, dtype=f32, device=d)
            self.h[mix] = torch.empty(V, CH, dtype=b16, device=d)
            self.rows[mix] = V
            prev = self.h[mix]
        self.inp["out"] = prev
        self.rows["out"] = V
        self.pred = torch.empty(V, OUT_PAD, dtype=f32, device=d)
        self.nvox = V
        # backward
        self.dpred = torch.empty(V, OUT_PAD, dtype=b16, device=d)
        self.dpredf = torch.empty(V, OUT_PAD, dtype=f32, device=d)
        big = V * CH
        self.dA = torch.empty(big, dtype=f32, device=d)
        self.dB = torch.empty(big, dtype=f32, device=d)
        self.dzb = torch.empty(big, dtype=b16, device=d)
        self.tA = torch.empty(max(big, self.spec.enc[-1] * _r16(B)), dtype=b16, device=d)
        self.tB = torch.empty(max(big, self.spec.enc[-1] * _r16(B)), dtype=b16, device=d)
        self.loss = torch.zeros(1, dtype=f32, device=d)

    # -- forward ------------------------------------------------------------------
    def forward(self, x):
        """x: [B, IN_PAD] float32 (normalised parameters) -> self.pred
        [B * ncell, OUT_PAD] in octree order."""
        nn = self.nn
        B = x.shape[0]
        self._alloc(B)
        nn.to_bf16(x.contiguous(), self.x0)
        a = self.x0
        for l in self.L[:4]:
            nn.gemm(a, self.W(l), bias=self.bias(l), act=l.act, zf=self.z[l.name], yb=self.h[l.name])
            a = self.h[l.name]
        for l in self.L[4:-1]:
            nn.gemm(self.inp[l.name], self.W(l), bias=self.bias(l), act=l.act, zf=self.z[l.name],
                    yb=self.h[l.name])
        lo = self.L[-1]
        nn.gemm(self.inp["out"], self.W(lo), bias=self.bias(lo), act=0, zf=self.pred)
        return self.pred

    # -- backward + update ----------------------------------------------------------
    def _wgrad(self, l, dzb, x, rows):
        """gW(l) += dz^T x over `rows` rows: both operands transposed so that
        the reduction (the rows) is the GEMM's contiguous K, split over CTAs."""
        nn = self.nn
        rp = _r16(rows)
        a = self.tA[:l.n * rp].view(l.n, rp)
        b = self.tB[:l.k * rp].view(l.k, rp)
        nn.transpose(dzb, a, rows_pad=rp)
        nn.transpose(x, b, rows_pad=rp)
        tiles = ((l.n + 127) // 128) * ((l.k + 255) // 256)
        splits = max(1, min(rp // 64, 296 // tiles))
        ks = max(64, (rp + splits - 1) // splits + 63) // 64 * 64
        nn.gemm(a, b, zf=self.gW(l), atomic=True, ksplit=ks)

    def backward(self, tgt, capture=None):
        """Gradients of the mean-squared error of self.pred against tgt
        [B * ncell, nvar] (normalised targets, octree order) into self.g.
        capture (a dict): receives per layer copies of the tensors its
        backward step consumed -- the BF16 pre-activation gradient (dzb),
        the FP32 one (dzf) and the BF16 layer input (x) -- and the input
        gradient it produced (dx, FP32), for layer-by-layer checks."""
        nn, torch = self.nn, self.torch
        self.g.zero_()
        self.loss.zero_()
        V = self.nvox
        nn.mse(self.pred, tgt, self.dpred, self.loss, gradf=self.dpredf)
        bufA, bufB = self.dA, self.dB
        dy = None
        for l in reversed(self.L):
            rows = self.rows.get(l.name, self.B)
            x = self.inp[l.name] if l.name in self.inp else self.h[f"enc{int(l.name[3:]) - 1}"]
            if l.name == "out":
                dzb, dzf = self.dpred, self.dpredf
            else:
                dy = dy.reshape(rows, l.n)   # the layer above returned it with its own row shape
                dzb = self.dzb[:rows * l.n].view(rows, l.n)
                dzf = bufB[:rows * l.n].view(rows, l.n)
                if l.act:
                    nn.silu_bwd(dy, self.z[l.name], dzb=dzb, dzf=dzf)
                else:
                    nn.to_bf16(dy, dzb)
                    dzf = dy
            self._wgrad(l, dzb, x, rows)
            nn.colsum(dzf, self.gb(l))
            if capture is not None:
                capture[l.name] = {"dzb": dzb.clone(), "dzf": dzf.clone(), "x": x.reshape(rows, l.k).clone()}
            if l.name == "enc1":
                break
            dx = bufA[:rows * l.k].view(rows, l.k)
            nn.gemm(dzb, self.WT(l), zf=dx)
            if capture is not None:
                capture[l.name]["dx"] = dx.clone()
            dy = dx
        return self.loss

    def adam(self, lr, wd=0.0):
        nn = self.nn
        self.step_n += 1
        for l in self.L:
            sl = slice(l.off, l.off + l.n * l.k)
            nn.adam(self.w[sl], self.g[sl], self.m[sl], self.v[sl], self.step_n, lr, wd=wd, w16=self.w16[sl],
                    w16t=self.w16t[sl], rows=l.n)
        b0 = self.L[0].boff
        sl = slice(b0, self.nparam)
        nn.adam(self.w[sl], self.g[sl], self.m[sl], self.v[sl], self.step_n, lr)

    def train(self, X, T, steps=2000, batch=16, lr=2e-3, seed=0, log_every=100):
        """X: [n, IN_PAD] float32, T: [n, ncell, nvar] float32 (device).
        Adam with a cosine learning-rate decay; returns [(step, loss)]."""
        torch = self.torch
        gen = torch.Generator().manual_seed(seed)
        n = X.shape[0]
        batch = min(batch, n)
        hist = []
        for s in range(steps):
            idx = torch.randperm(n, generator=gen)[:batch].to(self.dev)
            self.forward(X[idx])
            self.backward(T[idx].reshape(-1, self.spec.nvar))
            lr_s = lr * (0.05 + 0.95 * 0.5 * (1.0 + math.cos(math.pi * s / steps)))
            self.adam(lr_s)
            if (s + 1) % log_every == 0 or s == steps - 1:
                hist.append((s + 1, float(self.loss.item())))
        self.nn.error()
        return hist

    def predict(self, X):
        """[n, ncell, nvar] float32 (normalised, octree order)."""
        self.forward(X)
        self.nn.error()
        nv = self.spec.nvar
        return self.pred[:, :nv].reshape(X.shape[0], -1, nv)

    def state_dict(self):
        return {"w": self.w.detach().cpu().numpy()}

    def load_state_dict(self, d):
        self.w.copy_(self.torch.as_tensor(d["w"], device=self.dev))
        self._sync_bf16()


# ---- solver side: training data, prediction as a start, time to tolerance ----


def sample_params(n, seed, spec=BUMP):
    """[n, nparams] seeded uniform draws over the family's ranges (for the
    config-4 family: columns Mach, amplitude)."""
    rng = np.random.default_rng(seed)
    return np.stack([rng.uniform(lo, hi, size=n) for lo, hi in spec.ranges], axis=1)


def make_case(pv, seed=0, lusgs_fp32=False, ddadi=False, spec=BUMP):
    """The family's case at parameter values pv: (levels, prms, fs)."""
    from . import case
    kw = dict(zip(spec.params, [float(x) for x in pv]))
    levels, prms, fs = case.bump_case_mg(*spec.nodes, nlev=spec.nlev, mach=kw.get("mach", 0.5),
                                         amp=kw.get("amp", spec.amp), reynolds=spec.reynolds, h1=spec.h1,
                                         noise=spec.noise, seed=seed, inter=spec.inter, cfl=spec.cfl,
                                         cfll=spec.cfl, lusgs_fp32=lusgs_fp32, coarse_fp32=lusgs_fp32,
                                         turbulence=spec.turbulence, span_amp=spec.span_amp, zlen=spec.zlen)
    for q in prms:
        q.ddadi = int(ddadi)
        q.predgs_full = 1
    return levels, prms, fs


@dataclass
class Run:
    cycles: int
    seconds: float
    hist: np.ndarray            # per-cycle sum of squares of the density residual
    q: np.ndarray = field(default=None, repr=False)   # final interior targets [cells, nvar]


def solve(pv, cycles, init=None, tol=None, chunk=None, seed=0, keep_q=True, lusgs_fp32=False, ddadi=False,
          spec=BUMP):
    """Run the solver on the family's case at parameters pv for `cycles`
    cycles, or until the density residual's sum of squares is <= tol; init =
    solver state (TEMP, U, V, W, PDIFF[, RK, REPS]) of the fine interior
    cells to start from instead of the free stream; lusgs_fp32 runs every
    level's implicit stage in FP32, ddadi selects the DDADI implicit stage
    (LUSGS=0) instead of LU-SGS.  Wall time covers the cycles only (device
    synchronised)."""
    from .gpu import GpuSolver
    levels, prms, fs = make_case(pv, seed=seed, lusgs_fp32=lusgs_fp32, ddadi=ddadi, spec=spec)
    blk = levels[0]
    if init is not None:
        for n, v in init.items():
            blk.interior(n)[:] = v.reshape(blk.kmax, blk.jmax, blk.imax)
        if "RK" in init:   # the start-up's *OLD copies of k and omega
            blk.arrays["RKOLD"][:] = blk.arrays["RK"]
            blk.arrays["EPSOLD"][:] = blk.arrays["REPS"]
    chunk = chunk or (10 if tol is not None else 200)   # cycles per graph replay between residual checks
    g = GpuSolver(0)
    try:
        bid = g.add_levels(levels, prms) if len(levels) > 1 else g.add_block(blk, prms[0])
        for q in range(len(levels)):
            g.upload(bid + q)
        g.start(bid)
        g.sync()
        hs = []
        n = 0
        t0 = time.perf_counter()
        while n < cycles:
            m = min(chunk, cycles - n)
            h = g.cycles(m, bid, icycle0=n + 1)
            hs.append(h[:, 0])
            n += m
            if tol is not None and np.nanmin(h[:, 0]) <= tol:
                k = int(np.argmax(h[:, 0] <= tol))
                n = n - m + k + 1
                hs[-1] = h[:k + 1, 0]
                break
            if not np.isfinite(h[-1, 0]):
                break
        g.sync()
        sec = time.perf_counter() - t0
        q = None
        if keep_q:
            d = g.download(bid, list(QVARS[:spec.nvar]))
            q = np.stack([d[k].reshape(blk.kmax + 4, blk.jmax + 4, blk.imax + 4)[2:-2, 2:-2, 2:-2].ravel()
                          for k in QVARS[:spec.nvar]], axis=1)
        return Run(n, sec, np.concatenate(hs), q)
    finally:
        g.close()


class Dataset:
    """Normalised training targets in octree order and the statistics that
    undo the normalisation.  The conservative variables are scaled by each
    case's free-stream values; k and omega (7-variable families) enter as
    log(rho k / rho k_inf) and log(rho omega / rho omega_inf), which span
    the many decades between the wall and the free stream."""

    def __init__(self, P, qs, spec=BUMP):
        from .case import FlowConditions, sst_freestream
        self.spec = spec
        self.perm = octree_order(spec.root, spec.levels)
        self.P = np.asarray(P, dtype=float).reshape(len(qs), -1)
        sc = []
        for pv in self.P:
            fc, fs = self._fc(pv)
            s5 = freestream_scales(fs, fc.gamma, fc.rgas)
            if spec.nvar >= 7:
                rk, re = sst_freestream(fs)
                s5 = np.concatenate([s5, [rk, re]])
            sc.append(s5)
        self.scales = np.array(sc)
        y = np.stack([self._fwd(q[self.perm], s) for q, s in zip(qs, self.scales)])    # [n, ncell, nvar]
        self.mean = y.mean(axis=0)
        sd = (y - self.mean).reshape(-1, spec.nvar).std(axis=0)
        sd[3] = sd[2]                       # RW on the scale of RN
        self.std = np.maximum(sd, 1e-6)[None, :] * np.ones_like(self.mean)
        self.y = ((y - self.mean) / self.std).astype(np.float32)
        self.x = normalise_params(*self.P.T, spec=spec)

    def _fc(self, pv):
        from .case import FlowConditions
        kw = dict(zip(self.spec.params, pv))
        fc = FlowConditions(mach=float(kw.get("mach", 0.5)), reynolds=self.spec.reynolds)
        return fc, fc.freestream()

    def _fwd(self, q, s):
        y = q / s
        if self.spec.nvar >= 7:
            y[:, 5:7] = np.log(np.maximum(y[:, 5:7], 1e-30))
        return y

    def to_state(self, pred, pv):
        """Solver state of one prediction ([ncell, nvar] normalised, octree
        order) for the case at parameters pv."""
        fc, fs = self._fc(pv)
        s = freestream_scales(fs, fc.gamma, fc.rgas)
        y = pred * self.std + self.mean
        q = np.empty((len(self.perm), self.spec.nvar))
        if self.spec.nvar >= 7:
            from .case import sst_freestream
            rk, re = sst_freestream(fs)
            q[self.perm, :5] = y[:, :5] * s
            # k and omega kept inside the limits the solver itself applies:
            # LOLIM's free-stream floor (RKLIM, EPSLIM) and SUBIN's cap
            # RKMAX = FRSDEN FRSVEL^2 on rho k (ns3c.f:9742)
            q[self.perm, 5] = np.clip(np.exp(np.minimum(y[:, 5], 50.0)) * rk, rk, fs["rho"] * fs["u"] ** 2)
            q[self.perm, 6] = np.maximum(np.exp(np.minimum(y[:, 6], 60.0)) * re, re)
        else:
            q[self.perm] = y * s
        st = state_from_conservative(q, fs, fc.gamma, fc.rgas)
        # temperature and velocity inside the bounds the update limits keep
        # (TLOLIM / TUPLIM = 0.05 / 6 x FRSTEM) and twice the free-stream speed
        st["TEMP"] = np.minimum(st["TEMP"], 6.0 * fs["t"])
        vmax = 2.0 * fs["u"]
        for n in ("U", "V", "W"):
            st[n] = np.clip(st[n], -vmax, vmax)
        return st


def evaluate(net, data, P, tol_decades=2.0, max_cycles=3000, lusgs_fp32=True, ddadi_arms=False, spec=BUMP):
    """For each held-out case (rows of P): cycles and wall time to a residual
    tolerance
    * from the free stream with the plain FP64 solver (base),
    * from the free stream with the FP32 implicit stage (free32: what the
      precision form alone gains),
    * from the network's prediction with the FP32 implicit stage (warm).
    The tolerance is tol_decades below the free-stream start's first-cycle
    density residual (L2 norm), the same absolute level for every arm.  A
    run that does not reach it within max_cycles is reported as such: the
    plain solver stays the fallback.  ddadi_arms adds FP64 from the free
    stream and FP32 from the prediction with the DDADI implicit stage
    (LUSGS=0)."""
    import torch
    out = []
    for pv in np.asarray(P).reshape(len(P), -1):
        first = solve(pv, 1, keep_q=False, spec=spec)
        tol = first.hist[0] * 10.0 ** (-2.0 * tol_decades)
        base = solve(pv, max_cycles, tol=tol, keep_q=False, spec=spec)
        free32 = solve(pv, max_cycles, tol=tol, keep_q=False, lusgs_fp32=lusgs_fp32, spec=spec)
        t0 = time.perf_counter()
        pred = net.predict(torch.as_tensor(normalise_params(*[[x] for x in pv], spec=spec)).to(net.dev))
        st = data.to_state(pred[0].cpu().numpy(), pv)
        t_inf = time.perf_counter() - t0
        warm = solve(pv, max_cycles, init=st, tol=tol, keep_q=False, lusgs_fp32=lusgs_fp32, spec=spec)
        warm_reached = bool(np.isfinite(warm.hist).all() and warm.hist.min() <= tol)
        warm_cycles, warm_s = warm.cycles, warm.seconds + t_inf
        if not warm_reached:
            # the plain solver is the fallback: a start that fails costs its
            # own cycles plus the free-stream run (FP32 implicit stage)
            warm_cycles += free32.cycles
            warm_s += free32.seconds
        e = dict(params=[float(x) for x in pv], tol=float(tol),
                 base_cycles=base.cycles, base_s=base.seconds, base_reached=bool(base.hist.min() <= tol),
                 free32_cycles=free32.cycles, free32_s=free32.seconds,
                 free32_reached=bool(free32.hist.min() <= tol),
                 warm_cycles=warm_cycles, warm_s=warm_s, warm_reached=warm_reached, fallback=not warm_reached,
                 warm_start_decades=float(0.5 * np.log10(first.hist[0] / warm.hist[0])), infer_s=t_inf)
        if ddadi_arms:
            dbase = solve(pv, max_cycles, tol=tol, keep_q=False, ddadi=True, spec=spec)
            dwarm = solve(pv, max_cycles, init=st, tol=tol, keep_q=False, lusgs_fp32=True, ddadi=True, spec=spec)
            e.update(ddadi_base_cycles=dbase.cycles, ddadi_base_s=dbase.seconds,
                     ddadi_base_reached=bool(dbase.hist.min() <= tol),
                     ddadi_warm_cycles=dwarm.cycles, ddadi_warm_s=dwarm.seconds + t_inf,
                     ddadi_warm_reached=bool(dwarm.hist.min() <= tol))
        out.append(e)
    return out


def run_config(ntrain=64, ntest=16, cycles=2000, steps=6000, batch=16, lr=1e-3, tol_decades=2.0, seed_train=3,
               seed_test=4, log=print, ddadi_arms=False, spec=BUMP, max_cycles=None):
    """The learned-warm-start workload: solve ntrain seeded parameter points
    for `cycles` cycles as training data, train the network, then evaluate
    the ntest held-out points.  Returns a summary dict."""
    import torch
    t0 = time.perf_counter()
    Ptr = sample_params(ntrain, seed=seed_train, spec=spec)
    Pte = sample_params(ntest, seed=seed_test, spec=spec)
    runs = [solve(pv, cycles, spec=spec) for pv in Ptr]
    t_data = time.perf_counter() - t0
    log(f"training data: {ntrain} solves x {cycles} cycles in {t_data:.1f} s")
    # a diverged solve is no training field: keep the runs whose fields are
    # finite and whose density residual ends within 100x of its least value
    # (a solve that blew up after converging part-way ends far above it),
    # drop (and report) the others
    keep = [bool(np.isfinite(r.q).all() and np.isfinite(r.hist).all() and r.hist[-1] <= 100.0 * np.min(r.hist))
            for r in runs]
    dropped = [[float(x) for x in pv] for pv, k in zip(Ptr, keep) if not k]
    if dropped:
        log(f"training data: {len(dropped)} solves did not converge and are left out: {dropped}")
    if sum(keep) < 2:
        raise RuntimeError("warm start: fewer than two converged training solves")
    Ptr = Ptr[np.array(keep)]
    runs = [r for r, k in zip(runs, keep) if k]
    data = Dataset(Ptr, [r.q for r in runs], spec=spec)
    net = WarmStartNet(seed=0, spec=spec)
    X, T = torch.as_tensor(data.x).to(net.dev), torch.as_tensor(data.y).to(net.dev)
    t1 = time.perf_counter()
    hist = net.train(X, T, steps=steps, batch=batch, lr=lr, log_every=max(1, steps // 10))
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t1
    log(f"training: {steps} steps in {t_train:.1f} s, loss {hist}")
    ev = evaluate(net, data, Pte, tol_decades=tol_decades, max_cycles=max_cycles or max(3000, cycles),
                  ddadi_arms=ddadi_arms, spec=spec)
    base_s = sum(e["base_s"] for e in ev)
    warm_s = sum(e["warm_s"] for e in ev)
    free32_s = sum(e["free32_s"] for e in ev)
    out = dict(cases=ev, base_s=base_s, warm_s=warm_s, free32_s=free32_s, speedup=base_s / warm_s,
               network_gain=free32_s / warm_s,
               base_cycles=sum(e["base_cycles"] for e in ev), warm_cycles=sum(e["warm_cycles"] for e in ev),
               free32_cycles=sum(e["free32_cycles"] for e in ev),
               all_reached=all(e["base_reached"] and e["warm_reached"] and e["free32_reached"] for e in ev),
               fallbacks=sum(e["fallback"] for e in ev),
               loss=hist, t_data=t_data, t_train=t_train, steps=steps, ntrain=len(runs), ntest=ntest, cycles=cycles,
               dropped=dropped,
               family=spec.name, tol_decades=tol_decades)
    if ddadi_arms:
        for k in ("ddadi_base_s", "ddadi_warm_s", "ddadi_base_cycles", "ddadi_warm_cycles"):
            out[k] = sum(e[k] for e in ev)
        out["ddadi_reached"] = all(e["ddadi_base_reached"] and e["ddadi_warm_reached"] for e in ev)
    return out
