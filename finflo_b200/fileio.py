"""FINFLO's multi-block grid file (host-side I/O, not on the hot path).

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
