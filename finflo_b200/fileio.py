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
"""
from __future__ import annotations

import struct

import numpy as np


def _write_record(f, payload: bytes):
    n = struct.pack("<i", len(payload))
    f.write(n)
    f.write(payload)
    f.write(n)


def _read_record(f) -> bytes:
    head = f.read(4)
    if len(head) < 4:
        raise EOFError("grid file: unexpected end")
    (n,) = struct.unpack("<i", head)
    if n < 0:
        raise ValueError("grid file: record of more than 2 GiB (subrecords are not read)")
    payload = f.read(n)
    (m,) = struct.unpack("<i", f.read(4))
    if m != n or len(payload) != n:
        raise ValueError("grid file: record markers do not match")
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
