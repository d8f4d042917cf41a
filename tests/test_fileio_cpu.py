"""FINFLO's unformatted multi-block grid file (finflo_b200/fileio.py)."""
import struct

import numpy as np

from finflo_b200 import case, fileio, grid


def _blocks():
    X, Y, Z = grid.bump_nodes(17, 9, 9, h1=1e-3, amp=0.1)
    X2, Y2, Z2 = grid.box_nodes(np.linspace(0, 1, 5), np.linspace(0, 1, 3), np.linspace(0, 2, 9))
    return [(X, Y, Z), (X2, Y2, Z2)]


def test_layout_matches_the_fortran_records(tmp_path):
    """The exact bytes: 4-byte length markers around each record, NBLOCK,
    the node counts, then X, Y, Z of each block with i fastest."""
    path = tmp_path / "grid.bin"
    b = _blocks()
    fileio.write_grid(path, b)
    raw = path.read_bytes()
    assert struct.unpack("<3i", raw[:12]) == (4, 2, 4)
    assert struct.unpack("<8i", raw[12:44]) == (24, 17, 9, 9, 5, 3, 9, 24)
    n0 = 3 * 17 * 9 * 9 * 8
    (m,) = struct.unpack("<i", raw[44:48])
    assert m == n0
    x0 = np.frombuffer(raw[48:48 + 8 * 17], dtype="<f8")
    np.testing.assert_array_equal(x0, b[0][0][0, 0, :])


def test_round_trip_and_coarse_level(tmp_path):
    path = tmp_path / "grid.bin"
    b = _blocks()
    fileio.write_grid(path, b)
    back = fileio.read_grid(path)
    for (X, Y, Z), (Xr, Yr, Zr) in zip(b, back):
        for A, Ar in ((X, Xr), (Y, Yr), (Z, Zr)):
            np.testing.assert_array_equal(A, Ar)
    lev2 = fileio.read_grid(path, level=2)
    np.testing.assert_array_equal(lev2[0][0], b[0][0][::2, ::2, ::2])
    # the second block is three nodes long in j: that direction keeps every node
    np.testing.assert_array_equal(lev2[1][1], b[1][1][::2, :, ::2])


def test_block_from_a_grid_file_has_the_same_metrics(tmp_path):
    path = tmp_path / "grid.bin"
    X, Y, Z = grid.bump_nodes(17, 9, 9, h1=1e-3, amp=0.1)
    fileio.write_grid(path, [(X, Y, Z)])
    (Xr, Yr, Zr), = fileio.read_grid(path)
    fs = case.FlowConditions().freestream()
    a = case.new_block(X, Y, Z, case.channel_patches(16, 8, 8, fs))
    b = case.new_block(Xr, Yr, Zr, case.channel_patches(16, 8, 8, fs))
    for n in grid.METRIC_NAMES:
        np.testing.assert_array_equal(a.arrays[n], b.arrays[n])
