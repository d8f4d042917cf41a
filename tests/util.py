"""Shared helpers of the parity tests."""
import numpy as np

from finflo_b200 import case


def interior(blk, a):
    return a.reshape(blk.kmax + 4, blk.jmax + 4, blk.imax + 4)[2:-2, 2:-2, 2:-2]


def flux_scale(o, blk):
    """S = sum over the six faces of |F|/VOL per cell and variable (the
    normalisation of the 1e-12 residual parity criterion)."""
    import ctypes
    L = o.L
    nt = blk.ntot
    S = np.zeros((5, nt))
    istr = blk.imax + 4
    il = istr * (blk.jmax + 4)
    for d, st in ((1, 1), (2, istr), (3, il)):
        L.orc_flux_dir(o._b(), o._p(), d, 1)
        for v, n in enumerate(("F1R", "F1RM", "F1RN", "F1RW", "F1E")):
            F = np.abs(blk.arrays[n])
            S[v, :nt - st] += F[:nt - st] + F[st:]
    vol = blk.arrays["VOL"]
    return {n: interior(blk, S[v] / vol) for v, n in enumerate(("DRO", "DM", "DN", "DW", "DE"))}


def flux_scale_sst(o, blk):
    """S of the seven k-omega equations: face fluxes as in flux_scale plus
    the k and omega source terms."""
    L = o.L
    nt = blk.ntot
    names = ("F1R", "F1RM", "F1RN", "F1RW", "F1E", "F1RK", "F1EPS")
    S = np.zeros((7, nt))
    istr = blk.imax + 4
    il = istr * (blk.jmax + 4)
    for d, st in ((1, 1), (2, istr), (3, il)):
        L.orc_flux_dir_sst(o._b(), o._p(), d)
        for v, n in enumerate(names):
            F = np.abs(blk.arrays[n])
            S[v, :nt - st] += F[:nt - st] + F[st:]
    vol = blk.arrays["VOL"]
    out = {n: interior(blk, S[v] / vol) for v, n in enumerate(("DRO", "DM", "DN", "DW", "DE", "DRK", "DEPS"))}
    out["DRK"] = out["DRK"] + np.abs(interior(blk, blk.arrays["SRK"]))
    out["DEPS"] = out["DEPS"] + np.abs(interior(blk, blk.arrays["SEPS"]))
    return out


def momentum_floor(S):
    """Schemes whose momentum fluxes carry PDIFF rather than P (AUSM, KT): in
    a near-uniform field a cell's face fluxes of one momentum component can
    all vanish, and its S with them.  The three momentum components then
    share a floor of 1e-3 of the largest momentum scale in the block
    (hist_close does the same for the residual norms)."""
    fl = 1e-3 * max(S[m].max() for m in ("DM", "DN", "DW"))
    return {n: (np.maximum(v, fl) if n in ("DM", "DN", "DW") else v) for n, v in S.items()}


def make_pair(ni=17, nj=9, nk=9, **kw):
    bg, prm, fs = case.bump_case(ni, nj, nk, **kw)
    bc, _, _ = case.bump_case(ni, nj, nk, **kw)
    return bg, bc, prm, fs


def hist_close(got, ref, rtol):
    """Residual-norm histories (sums of squares of DRO, DM, DN, DW, DE): in
    spanwise-uniform cases one momentum residual is zero up to rounding, so
    the three momentum components share one scale."""
    got, ref = np.asarray(got), np.asarray(ref)
    mom = np.abs(ref[:, 1:4]).max()
    for c in range(5):
        atol = rtol * mom if c in (1, 2, 3) else 0.0
        np.testing.assert_allclose(got[:, c], ref[:, c], rtol=rtol, atol=atol)
