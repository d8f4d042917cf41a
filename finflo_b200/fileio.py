"""FINFLO's multi-block grid file, restart file RSTART and boundary-condition
file (host-side I/O, not on the hot path).

The file is Fortran unformatted sequential (main.f:1366-1374, GRIMP
messp.f:1079-1127): a record with NBLOCK, a record with (IX, IY, IZ) of
every block (node counts), then one record per block with X, Y and Z of its
IX*IY*IZ nodes, i fastest.  Integers are 4 bytes and reals 8 (the reference
is built with -r8 / -fdefault-real-8); every record is framed by its byte
length as a 4-byte integer before and after it.

Reading a coarser multigrid level takes every 2^(LEVEL-1)-th node per
direction, except in a direction three nodes long (k: three or fewer),
which keeps every node (GRIMP messp.f:1091-1096).

The restart file RSTART (WRITRS outp3.f:2042, READRS outp3.f:1119) is
unformatted sequential too: a record with the flags TIMEL, COORL, CHIMEL
(4-byte Fortran logicals), then per block one record per variable over all
NNMAX = (IMAX+4)(JMAX+4)(KMAX+4) cells, ghost cells included.  The state is
stored as U, V, W, temperature and PDIFF = P - FRSPRE (no conservative
variables); the start-up after READRS rebuilds P (ns3c.f:341) and STATIM
the rest.  This module writes and reads the records of the variants this
path runs: no scalars (NSCAL=0), no transition or multiphase variables, no
Reynolds stresses, IPRESC=0 without FRESUL, and neither deforming nor
chimera grids.
"""
from __future__ import annotations

import math
import struct

import numpy as np


def _write_record(f, payload: bytes):
    n = struct.pack("<i", len(payload))
    f.write(n)
    f.write(payload)
    f.write(n)


def _read_record(f, label="grid file") -> bytes:
    """One unformatted sequential record; `label` names the file kind in the
    error messages (grid file, RSTART)."""
    head = f.read(4)
    if len(head) < 4:
        raise EOFError(f"{label}: unexpected end")
    (n,) = struct.unpack("<i", head)
    if n < 0:
        raise ValueError(f"{label}: record of more than 2 GiB (subrecords are not read)")
    payload = f.read(n)
    tail = f.read(4)
    if len(payload) != n or len(tail) < 4:
        raise EOFError(f"{label}: unexpected end inside a record")
    (m,) = struct.unpack("<i", tail)
    if m != n:
        raise ValueError(f"{label}: record markers do not match")
    return payload


def write_grid(path, blocks):
    """blocks: list of (X, Y, Z) node arrays of shape (IZ, IY, IX)."""
    with open(path, "wb") as f:
        _write_record(f, struct.pack("<i", len(blocks)))
        dims = []
        for X, Y, Z in blocks:
            iz, iy, ix = X.shape
            dims += [ix, iy, iz]
        _write_record(f, struct.pack(f"<{len(dims)}i", *dims))
        for X, Y, Z in blocks:
            buf = np.concatenate([np.asarray(A, dtype="<f8").ravel() for A in (X, Y, Z)])
            _write_record(f, buf.tobytes())


def read_grid(path, level=1):
    """The blocks' (X, Y, Z) node arrays, shape (IZ, IY, IX), at multigrid
    level `level` (1 = the file's own nodes)."""
    with open(path, "rb") as f:
        (nblock,) = struct.unpack("<i", _read_record(f))
        dims = struct.unpack(f"<{3 * nblock}i", _read_record(f))
        blocks = []
        step = 2 ** (level - 1)
        for n in range(nblock):
            ix, iy, iz = dims[3 * n:3 * n + 3]
            ngrid = ix * iy * iz
            a = np.frombuffer(_read_record(f), dtype="<f8")
            if a.size != 3 * ngrid:
                raise ValueError(f"grid file: block {n + 1} has {a.size} values, expected {3 * ngrid}")
            si = 1 if ix == 3 else step
            sj = 1 if iy == 3 else step
            sk = 1 if iz <= 3 else step
            if (ix - 1) % si or (iy - 1) % sj or (iz - 1) % sk:
                raise ValueError(f"grid file: block {n + 1} does not coarsen to level {level}")
            XYZ = [a[c * ngrid:(c + 1) * ngrid].reshape(iz, iy, ix)[::sk, ::sj, ::si].copy() for c in range(3)]
            blocks.append(tuple(XYZ))
        return blocks


# WRITRS outp3.f:2095-2115: the per-block records, in file order.  With
# IPRESC=0 and no FRESUL the three PRC records repeat DDEPS, PDIFF and TEMP.
RESTART_FIELDS = ("U", "V", "W", "EPS2", "VIST", "OHMI", "RK", "REPS", "PTUR",
                  "DDEPS", "PDIFF", "TEMP", "DDEPS", "PDIFF", "TEMP")
# WRITRS outp3.f:2299-2341 (TIMEL): the previous time level, then the running
# time averages (first and second moments).
RESTART_TIME_FIELDS = ("ROLE2", "RMLE2", "RNLE2", "RWLE2", "RKLE2", "EPSLE2", "ELE2",
                       "ROAV1", "RMAV1", "RNAV1", "RWAV1", "RKAV1", "EPSAV1", "EAV1",
                       "ROAV2", "RMAV2", "RNAV2", "RWAV2", "PAV1", "TAV1", "EAV2",
                       "RUVAV", "RUWAV", "RVWAV")


def write_restart(path, blocks, *, timel=False):
    """Write RSTART.  blocks: list of dicts, variable name -> the block's
    NNMAX values; a variable the dict lacks (DDEPS, the time averages) is
    written as zeros, as a block that never accumulated it holds."""
    with open(path, "wb") as f:
        _write_record(f, struct.pack("<3i", int(bool(timel)), 0, 0))
        sizes = [_block_size(d) for d in blocks]
        for names in (RESTART_FIELDS,) + ((RESTART_TIME_FIELDS,) if timel else ()):
            for d, n in zip(blocks, sizes):
                for name in names:
                    a = d.get(name)
                    a = np.zeros(n) if a is None else np.asarray(a, dtype="<f8").ravel()
                    if a.size != n:
                        raise ValueError(f"restart: {name} has {a.size} values, expected {n}")
                    _write_record(f, a.tobytes())


def _block_size(d):
    for a in d.values():
        return np.asarray(a).size
    raise ValueError("restart: a block without variables")


def read_restart(path, sizes, *, timel=False):
    """Read RSTART.  sizes: NNMAX of each block (the file holds no
    dimensions; READRS takes them from the grid).  Returns (time_level,
    blocks): the file's TIMEL flag and per block a dict of its variables.
    The time-level records are read only when both the file and `timel`
    have them (READRS outp3.f:1483, IF(TIMEL .AND. TIME2))."""
    with open(path, "rb") as f:
        flags = _read_record(f, "restart")
        if len(flags) != 12:
            raise ValueError("restart: the first record is not TIMEL, COORL, CHIMEL")
        time2, coor2, chime2 = struct.unpack("<3i", flags)
        if coor2 or chime2:
            raise ValueError("restart: deforming-grid and chimera restarts are not read")
        out = [dict() for _ in sizes]
        groups = (RESTART_FIELDS,) + ((RESTART_TIME_FIELDS,) if (timel and time2) else ())
        for names in groups:
            for d, n in zip(out, sizes):
                for name in names:
                    a = np.frombuffer(_read_record(f, "restart"), dtype="<f8")
                    if a.size != n:
                        raise ValueError(f"restart: {name} has {a.size} values, expected {n}")
                    d[name] = a.copy()
        return bool(time2), out


def block_restart_vars(blk, *, timel=False):
    """The restart variables a block holds (views of its arrays)."""
    names = RESTART_FIELDS + (RESTART_TIME_FIELDS if timel else ())
    return {n: blk.arrays[n] for n in dict.fromkeys(names) if n in blk.arrays}


def load_restart_vars(blk, d):
    """Copy a block's restart variables into its arrays.  The conservative
    state follows from them at start-up: BOUNDI's STATIM rebuilds RO, RM,
    RN, RW and E from U, V, W, TEMP and PDIFF."""
    for n, a in d.items():
        if n in blk.arrays:
            if a.size != blk.arrays[n].size:
                raise ValueError(f"restart: {n} has {a.size} values, the block {blk.arrays[n].size}")
            blk.arrays[n][:] = a.reshape(blk.arrays[n].shape)


# ---- boundary-condition file (READBC gluebm.f:2553) ------------------------
#
# Formatted text: a title line, NBLKS, then per block a comment line, its
# cell counts IDIM JDIM KDIM and six faces, each "IFACE NOFBCS" followed by
# NOFBCS patch lines "<TYP> <numbers and letters>".  Per patch type:
#   CON / PER (1:1, PER = periodic, ICON(20) = 1): r1a r1b r2a r2b, the
#       neighbour block, its face and its patch number on that face (the
#       patch's position in its face's list);
#   INL / OUT: the INLOUT sub-type (ICON(8) = ICON(27)); a type <= 10 or in
#       21..30 is followed by one line with the boundary-value file name;
#   SOL / ROT / MOV: force-group letters (FGIDS, blanked out before the
#       numbers are read), then one extra line "IHEAT RCON(1..14)" (13 reals
#       leave RCON(14) = WTRAN = 1);
#   any non-connective patch on a face with several patches: r1a r1b r2a r2b.
# A face with one patch always covers the whole face (the ranges are reset).
# Numbers are read as INLINE/UNWRAP read them (gluebm.f:3789, 3856): runs of
# digits, '.' and '-' between any other characters, rounded to integers.
# READBC then replaces each connection's neighbour patch number by that
# patch's ranges (gluebm.f:3192-3228, the completion loop) and mirrors the
# MIR data (3232-3250).

BC_TYPES = {"DUM": 0, "CON": 1, "PER": 1, "EXT": 2, "INL": 3, "MIR": 4, "OUT": 5, "CYC": 6, "SNG": 7, "SOL": 8,
            "ROT": 9, "MOV": 10, "SLD": 11, "CHI": 12, "FRE": 13, "MIX": 14, "HTS": 15, "SLI": 16, "INP": 17,
            "CML": 1, "ACT": 1}
_CONNECTIVE = ("CON", "PER", "CYC", "HTS", "SLD", "MIX")


class BcPatch:
    """One patch of the BC file with the ICON columns READBC fills (1-based
    block and patch numbers, as in the file)."""

    def __init__(self, kind, block, iface, local):
        self.kind = kind                  # the three letters as written
        self.ityp = BC_TYPES[kind]        # ICON(1)
        self.block = block                # ICON(2)
        self.iface = iface                # ICON(3)
        self.local = local                # ICON(14): position on its face
        self.r1a = self.r1b = self.r2a = self.r2b = 0   # ICON(4..7)
        self.nblock = self.nface = self.npatch = 0      # ICON(8), (9), (10) as read
        self.n1a = self.n1b = self.n2a = self.n2b = 0   # neighbour ranges, after completion
        self.partner = -1                 # ICON(15): global index of the matching patch
        self.itype = 0                    # INL/OUT: INLOUT sub-type, ICON(27)
        self.iheat = 0                    # ICON(20): SOL heat condition, PER = 1
        self.rcon = [0.0] * 14            # SOL extra line RCON(1..14)
        self.groups = ""                  # force-group letters
        self.bfile = ""                   # INL/OUT boundary-value file name


def _numbers(s, nv):
    """INLINE/UNWRAP: up to nv integers from s (NINT of each number)."""
    out, i, n = [], 0, len(s)
    num = set("0123456789.-")
    while len(out) < nv:
        while i < n and s[i] not in num:
            i += 1
        ifun = des = ddes = 0
        neg, acc = 1, False
        while i < n and s[i] in num:
            c = s[i]
            if c == ".":
                ddes = 1
            elif c == "-":
                neg = -1
            else:
                ifun = ifun * 10 + int(c)
                des += ddes
                acc = True
            i += 1
        if not acc:
            break
        v = neg * ifun / 10 ** des
        out.append(int(math.floor(v + 0.5)) if v >= 0 else -int(math.floor(-v + 0.5)))
    return out


def _face_cells(iface, dims):
    i, j, k = dims
    return {1: (j, k), 4: (j, k), 2: (i, k), 5: (i, k), 3: (i, j), 6: (i, j)}[iface]


def read_bc(path, dims=None):
    """Read a BC file.  dims: the blocks' cell counts (IMAX, JMAX, KMAX)
    from the grid file, checked against the file's.  Returns the patches
    in file order with their connections completed."""
    with open(path) as f:
        lines = f.read().splitlines()
    pos = [0]

    def nxt():
        if pos[0] >= len(lines):
            raise ValueError("BC file: unexpected end")
        pos[0] += 1
        return lines[pos[0] - 1]

    nxt()   # title
    nblk = int(nxt().split()[0])
    if dims is not None and nblk != len(dims):
        raise ValueError(f"BC file: {nblk} blocks, the grid has {len(dims)}")
    patches, bdims = [], []
    for ib in range(1, nblk + 1):
        nxt()
        d = tuple(int(x) for x in nxt().split()[:3])
        if dims is not None and tuple(dims[ib - 1]) != d:
            d = tuple(dims[ib - 1])   # READBC falls back to the grid's dimensions
        bdims.append(d)
        for _ in range(6):
            iface, nof = (int(x) for x in nxt().split()[:2])
            if iface < 1 or iface > 6:
                raise ValueError(f"BC file: illegal face number {iface} in block {ib}")
            covered = 0
            for j in range(1, nof + 1):
                line = nxt().lstrip()
                kind, rest = line[:3], line[3:]
                if kind not in BC_TYPES:
                    raise ValueError(f"BC file: unknown boundary condition {kind!r} in block {ib}")
                p = BcPatch(kind, ib, iface, j)
                if p.kind == "PER":
                    p.iheat = 1
                if kind in ("SOL", "ROT", "MOV", "HTS", "SLI", "CML", "INL", "OUT", "ACT"):
                    p.groups = "".join(c for c in rest if c.isalpha() and c.isascii())
                    rest = "".join(" " if (c.isalpha() and c.isascii()) else c for c in rest)
                if kind in _CONNECTIVE:
                    v = _numbers(rest, 8)
                    if len(v) < 7:
                        raise ValueError(f"BC file: automatic connections (AUTOCON) are not read: block {ib}")
                    p.r1a, p.r1b, p.r2a, p.r2b, p.nblock, p.nface, p.npatch = v[:7]
                elif kind in ("INL", "OUT"):
                    if nof > 1:
                        raise ValueError("BC file: an inlet or outlet must cover the whole block face")
                    v = _numbers(rest, 1)
                    p.itype = v[0] if v else 1
                    if p.itype <= 10 or 20 < p.itype <= 30:
                        p.bfile = nxt().strip()
                if nof == 1:
                    a, b = _face_cells(iface, d)
                    p.r1a, p.r1b, p.r2a, p.r2b = 1, a, 1, b
                elif kind not in _CONNECTIVE and kind != "MOV":
                    v = _numbers(rest, 4)
                    if len(v) != 4:
                        raise ValueError(f"BC file: patch ranges missing in block {ib}, face {iface}")
                    p.r1a, p.r1b, p.r2a, p.r2b = v
                if kind in ("SOL", "ROT", "MOV"):
                    extra = nxt().split()
                    p.iheat = int(float(extra[0]))
                    vals = [float(x) for x in extra[1:15]]
                    if len(vals) == 13:
                        vals.append(1.0)   # WTRAN = 1: fully turbulent
                    if len(vals) != 14:
                        raise ValueError(f"BC file: the solid-wall line of block {ib} lacks values")
                    p.rcon = vals
                covered += (p.r1b - p.r1a + 1) * (p.r2b - p.r2a + 1)
                patches.append(p)
            a, b = _face_cells(iface, d)
            if covered != a * b:
                raise ValueError(f"BC file: the patches of block {ib}, face {iface} do not cover it")
    _complete_connections(patches)
    return patches, bdims


def _complete_connections(patches):
    """gluebm.f:3192-3228: a connection's (neighbour block, face, patch
    number) -> the neighbour patch's ranges and index; the areas must
    match.  Mirror patches point at themselves (3232-3250)."""
    for i, p in enumerate(patches):
        if p.ityp in (4, 12, 13):
            p.nblock, p.nface = p.block, p.iface
            p.n1a, p.n1b, p.n2a, p.n2b = p.r1a, p.r1b, p.r2a, p.r2b
            p.partner = i
            continue
        if p.kind not in _CONNECTIVE:
            continue
        for j, q in enumerate(patches):
            if q.kind in _CONNECTIVE and q.block == p.nblock and q.iface == p.nface and q.local == p.npatch:
                if (p.r1b - p.r1a + 1) * (p.r2b - p.r2a + 1) != (q.r1b - q.r1a + 1) * (q.r2b - q.r2a + 1):
                    raise ValueError(f"BC file: the areas of the connection block {p.block}, face {p.iface} "
                                     "do not match")
                p.n1a, p.n1b, p.n2a, p.n2b = q.r1a, q.r1b, q.r2a, q.r2b
                p.partner = j
                break
        else:
            raise ValueError(f"BC file: no partner for the connection of block {p.block}, face {p.iface}")


def write_bc(path, dims, patches, title="FINFLO boundary conditions"):
    """Write a BC file for blocks of cell counts dims; patches as read_bc
    returns them (a face's patches in their `local` order)."""
    out = [title, f"{len(dims)}"]
    for ib, d in enumerate(dims, start=1):
        out += [f"block {ib}", f"{d[0]} {d[1]} {d[2]}"]
        for iface in range(1, 7):
            mine = sorted((p for p in patches if p.block == ib and p.iface == iface), key=lambda p: p.local)
            out.append(f"{iface} {len(mine)}")
            for p in mine:
                if p.kind in _CONNECTIVE:
                    out.append(f"{p.kind} {p.r1a} {p.r1b} {p.r2a} {p.r2b} {p.nblock} {p.nface} {p.npatch}")
                elif p.kind in ("INL", "OUT"):
                    out.append(f"{p.kind} {p.itype} {p.groups}".rstrip())
                    if p.itype <= 10 or 20 < p.itype <= 30:
                        out.append(p.bfile or "BOUNDARY.DAT")
                else:
                    rng = f" {p.r1a} {p.r1b} {p.r2a} {p.r2b}" if len(mine) > 1 else ""
                    out.append(f"{p.kind}{rng} {p.groups}".rstrip())
                if p.kind in ("SOL", "ROT", "MOV"):
                    out.append(f"{p.iheat} " + " ".join(repr(float(x)) for x in p.rcon))
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")
