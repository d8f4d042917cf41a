"""FINFLO's unformatted multi-block grid file and restart file RSTART
(finflo_b200/fileio.py)."""
import struct

import numpy as np
import pytest

from finflo_b200 import case, fileio, grid
from oracle.oracle import Oracle


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


def test_restart_record_layout(tmp_path):
    """RSTART: the flags record (three 4-byte logicals), then per block the
    fifteen NNMAX records of WRITRS in order, DDEPS written as zeros."""
    blk, prm, fs = case.bump_case(9, 7, 5)
    path = tmp_path / "RSTART"
    fileio.write_restart(path, [fileio.block_restart_vars(blk)])
    raw = path.read_bytes()
    assert struct.unpack("<5i", raw[:20]) == (12, 0, 0, 0, 12)
    n = blk.ntot
    rec = 8 * n + 8
    assert len(raw) == 20 + 15 * rec
    for k, name in enumerate(fileio.RESTART_FIELDS):
        off = 20 + k * rec
        assert struct.unpack("<i", raw[off:off + 4]) == (8 * n,)
        a = np.frombuffer(raw[off + 4:off + 4 + 8 * n], dtype="<f8")
        want = blk.arrays[name].ravel() if name in blk.arrays else np.zeros(n)
        np.testing.assert_array_equal(a, want)


def test_restart_round_trip_timel(tmp_path):
    """Two blocks with the time-level records; a reader without TIMEL stops
    after the main records, as READRS does."""
    blocks = []
    for dims in ((9, 7, 5), (5, 5, 3)):
        blk, prm, fs = case.bump_case(*dims, turbulence="sst", reynolds=1e6)
        rng = np.random.default_rng(dims[0])
        for n in ("ROLE2", "RMLE2", "ELE2"):
            blk.arrays[n][:] = rng.standard_normal(blk.ntot)
        blocks.append(blk)
    path = tmp_path / "RSTART"
    fileio.write_restart(path, [fileio.block_restart_vars(b, timel=True) for b in blocks], timel=True)
    time2, got = fileio.read_restart(path, [b.ntot for b in blocks], timel=True)
    assert time2
    for b, d in zip(blocks, got):
        for n in ("U", "TEMP", "PDIFF", "RK", "REPS", "VIST", "ROLE2", "RMLE2", "ELE2"):
            np.testing.assert_array_equal(d[n], b.arrays[n].ravel())
        assert not d["DDEPS"].any() and not d["RVWAV"].any()
    time2, got = fileio.read_restart(path, [b.ntot for b in blocks])
    assert time2 and "ROLE2" not in got[0]
    with pytest.raises(ValueError):
        fileio.read_restart(path, [blocks[0].ntot + 1, blocks[1].ntot])


@pytest.mark.parametrize("sst", [False, True])
def test_restart_continues_the_run(tmp_path, sst):
    """Ten cycles, RSTART, a fresh case read from it and started as usual,
    five more cycles: the residual history equals fifteen cycles in one run
    (every cycle starts with STATIM, which rebuilds the conservative state
    from the primitive variables the file holds)."""
    kw = dict(turbulence="sst", reynolds=1e6, mach=0.6, h1=1e-4) if sst else {}
    blk, prm, fs = case.bump_case(17, 9, 9, **kw)
    o = Oracle(blk, prm)
    o.start()
    full = [o.cycle(i + 1)[0] for i in range(15)]
    blk, prm, fs = case.bump_case(17, 9, 9, **kw)
    o = Oracle(blk, prm)
    o.start()
    for i in range(10):
        o.cycle(i + 1)
    path = tmp_path / "RSTART"
    fileio.write_restart(path, [fileio.block_restart_vars(blk)])
    blk2, prm2, fs2 = case.bump_case(17, 9, 9, **kw)
    _, got = fileio.read_restart(path, [blk2.ntot])
    fileio.load_restart_vars(blk2, got[0])
    o2 = Oracle(blk2, prm2)
    o2.start()
    rest = [o2.cycle(i + 11)[0] for i in range(5)]
    np.testing.assert_allclose(np.array(rest), np.array(full[10:]), rtol=1e-9)


@pytest.mark.parametrize("flags", [(0, 1, 0), (0, 0, 1)])
def test_restart_rejects_deforming_and_chimera_files(tmp_path, flags):
    """A file whose COORL or CHIMEL flag is set holds records this path does
    not read; the reader refuses it instead of misreading what follows."""
    path = tmp_path / "RSTART"
    with open(path, "wb") as f:
        fileio._write_record(f, struct.pack("<3i", *flags))
    with pytest.raises(ValueError, match="chimera"):
        fileio.read_restart(path, [10])


def test_restart_truncated_file_names_the_restart(tmp_path):
    """A truncated RSTART is reported as a restart error, not a grid error."""
    blk, prm, fs = case.bump_case(9, 7, 5)
    path = tmp_path / "RSTART"
    fileio.write_restart(path, [fileio.block_restart_vars(blk)])
    data = path.read_bytes()
    path.write_bytes(data[:len(data) - 100])
    with pytest.raises((EOFError, ValueError), match="restart"):
        fileio.read_restart(path, [blk.ntot])


def _timel_steps(o, steps, inner, first_step=0, hist=None):
    for s in range(first_step, first_step + steps):
        if s:
            o.time_levels(1)   # NEWTIM at the start of every later physical step
        for i in range(inner):
            r = o.cycle(i + 1)[0]
            if hist is not None:
                hist.append(r)


def test_restart_continues_a_timel_run(tmp_path):
    """Time-accurate run: two physical steps, RSTART with the time-level
    records (written at the end of a step, as WRITRS is), a fresh case read
    from it whose next step begins with NEWTIM; its third step equals the
    third step of the uninterrupted run."""
    inner, dt = 8, 2e-5
    blk, prm, fs = case.bump_case(17, 9, 9)
    prm.timel, prm.dt = 1, dt
    o = Oracle(blk, prm)
    o.start()
    o.time_levels(0)   # STARTI
    full = []
    _timel_steps(o, 3, inner, hist=full)

    blk, prm, fs = case.bump_case(17, 9, 9)
    prm.timel, prm.dt = 1, dt
    o = Oracle(blk, prm)
    o.start()
    o.time_levels(0)
    _timel_steps(o, 2, inner)
    path = tmp_path / "RSTART"
    fileio.write_restart(path, [fileio.block_restart_vars(blk, timel=True)], timel=True)

    blk2, prm2, fs2 = case.bump_case(17, 9, 9)
    prm2.timel, prm2.dt = 1, dt
    time2, got = fileio.read_restart(path, [blk2.ntot], timel=True)
    assert time2
    fileio.load_restart_vars(blk2, got[0])
    o2 = Oracle(blk2, prm2)
    o2.start()
    rest = []
    _timel_steps(o2, 1, inner, first_step=2, hist=rest)
    np.testing.assert_allclose(np.array(rest), np.array(full[2 * inner:]), rtol=1e-9)
