"""FINFLO's boundary-condition file (READBC gluebm.f:2553): reading, the
connection completion, writing, and a case read from a grid file and a BC
file running like the case built in memory."""
import numpy as np
import pytest

from finflo_b200 import case, fileio, grid
from oracle.oracle import Oracle

FIELDS = ["ityp", "iface", "r1a", "r1b", "r2a", "r2b", "ibtype", "iheat", "nface", "n1a", "n2a"]


def _multiblock():
    it = case.bump_multiblock_blocks(cells=(32, 16, 8), nb=(2, 2, 2), nlev=1, turbulence=None)
    _, fs = next(it)
    blocks = [lv[0] for lv, _ in it]
    return blocks, fs


def test_round_trip_of_a_multiblock_case(tmp_path):
    """Eight blocks with inlet, outlet, walls, interior 1:1 cuts and the
    periodic z faces: written, read back and turned into patch tables, every
    ICON field the library reads is unchanged."""
    blocks, fs = _multiblock()
    pats = [b.patches for b in blocks]
    dims = [b.dims for b in blocks]
    path = tmp_path / "BC"
    fileio.write_bc(path, dims, case.bc_from_patches(pats, periodic_faces=(3, 6)))
    bc, d2 = fileio.read_bc(path, dims)
    assert d2 == dims
    assert sum(p.kind == "PER" for p in bc) == 16
    back = case.patches_from_bc(bc, len(blocks), fs)
    for pa, pb in zip(pats, back):
        assert len(pa) == len(pb)
        for a, b in zip(pa, pb):
            for f in FIELDS:
                assert getattr(a, f) == getattr(b, f), f


HAND = """Two blocks, hand written
2
 block one
  8 4 2
1 1
 INL 4  A
inlet.dat
2 2
 SOL 1 4 1 2 AB
1 300.0 0 0 0 0 0 0 0 0 0 0 0 0
 MIR 5 8 1 2
3 1
 PER 1 8 1 4 1 6 1
4 1
 CON 1 4 1 2 2 1 1
5 1
 SOL
0 0 0 0 0 0 0 0 0 0 0 0 0 0 0.5
6 1
 PER 1 8 1 4 1 3 1
  block two
  6 4 2
1 1
 CON 1 4 1 2 1 4 1
2 1
 SOL
0 0 0 0 0 0 0 0 0 0 0 0 0 0 1
3 1
 MIR
4 1
 OUT 3
outlet.dat
5 1
 SOL
0 0 0 0 0 0 0 0 0 0 0 0 0 0 1
6 1
 MIR
"""


def test_reads_a_hand_written_file(tmp_path):
    path = tmp_path / "BC"
    path.write_text(HAND)
    bc, dims = fileio.read_bc(path, [(8, 4, 2), (6, 4, 2)])
    assert len(bc) == 13
    inl = bc[0]
    assert (inl.kind, inl.itype, inl.bfile, inl.groups) == ("INL", 4, "inlet.dat", "A")
    sol = bc[1]
    assert (sol.r1a, sol.r1b, sol.r2a, sol.r2b, sol.iheat, sol.groups) == (1, 4, 1, 2, 1, "AB")
    assert sol.rcon[0] == 300.0 and sol.rcon[13] == 1.0     # 13 reals: WTRAN defaults to 1
    mir = bc[2]
    assert (mir.kind, mir.r1a, mir.r1b) == ("MIR", 5, 8)
    assert (mir.nblock, mir.nface, mir.partner) == (1, 2, 2)   # a mirror points at itself
    per = bc[3]
    assert per.iheat == 1 and per.nblock == 1 and per.nface == 6 and per.partner == 6
    con = bc[4]
    assert (con.nblock, con.nface, con.n1a, con.n1b, con.n2a, con.n2b) == (2, 1, 1, 4, 1, 2)
    assert bc[5].rcon[13] == 0.5
    assert bc[10].kind == "OUT" and bc[10].itype == 3 and bc[10].bfile == "outlet.dat"
    fs = case.FlowConditions().freestream()
    tables = case.patches_from_bc(bc, 2, fs)
    assert [p.ityp for p in tables[0]] == [grid.BC_INL, grid.BC_SOL, grid.BC_MIR, grid.BC_CON, grid.BC_CON,
                                           grid.BC_SOL, grid.BC_CON]
    assert tables[0][4].ibtype == 1 and tables[1][0].ibtype == 0


@pytest.mark.parametrize("edit,msg", [
    (lambda s: s.replace(" MIR 5 8 1 2", " MIR 5 7 1 2"), "do not cover"),
    (lambda s: s.replace(" CON 1 4 1 2 2 1 1", " CON 1 4 1 2 2 1 2"), "no partner"),
    (lambda s: s.replace(" CON 1 4 1 2 1 4 1", " CON 1 4 1 1 1 4 1").replace("  6 4 2\n1 1", "  6 4 2\n1 2")
     .replace(" CON 1 4 1 1 1 4 1\n", " CON 1 4 1 1 1 4 1\n MIR 1 4 2 2\n"), "areas"),
    (lambda s: s.replace(" OUT 3", " XYZ 3"), "unknown boundary condition"),
    (lambda s: s.replace(" CON 1 4 1 2 2 1 1", " CON 1 4 1 2"), "AUTOCON"),
])
def test_refuses_broken_files(tmp_path, edit, msg):
    path = tmp_path / "BC"
    path.write_text(edit(HAND))
    with pytest.raises(ValueError, match=msg):
        fileio.read_bc(path, [(8, 4, 2), (6, 4, 2)])


def test_case_from_grid_and_bc_files_runs_like_the_built_case(tmp_path):
    """The bump channel written as a grid file and a BC file, read back,
    set up and run: the oracle's residual history equals the in-memory
    case's."""
    blk, prm, fs = case.bump_case(17, 9, 9)
    X, Y, Z = blk.nodes
    fileio.write_grid(tmp_path / "GRID", [(X, Y, Z)])
    fileio.write_bc(tmp_path / "BC", [blk.dims], case.bc_from_patches([blk.patches]))
    (X2, Y2, Z2), = fileio.read_grid(tmp_path / "GRID")
    dims = [(X2.shape[2] - 1, X2.shape[1] - 1, X2.shape[0] - 1)]
    bc, _ = fileio.read_bc(tmp_path / "BC", dims)
    blk2 = case.new_block(X2, Y2, Z2, case.patches_from_bc(bc, 1, fs)[0])
    case.init_freestream(blk2, fs, noise=1e-3, seed=0)
    h = []
    for b in (blk, blk2):
        o = Oracle(b, prm)
        o.start()
        h.append(np.array([o.cycle(i + 1)[0] for i in range(5)]))
    np.testing.assert_array_equal(h[0], h[1])
