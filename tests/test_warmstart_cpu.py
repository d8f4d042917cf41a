"""Host-side pieces of the learned warm start: octree order of the decoder's
voxels, the layer table, and the conversion of predicted conservative
variables to the solver's state."""
import numpy as np

from finflo_b200 import case, warmstart as ws


def test_octree_order_is_a_permutation_with_parent_child_nesting():
    o = ws.octree_order()
    ni, nj, nk = ws.GRID
    assert sorted(o.tolist()) == list(range(ni * nj * nk))
    i, j, k = o % ni, (o // ni) % nj, o // (ni * nj)
    # voxel v at the finest level has parent v // 8 one level up: the coarse
    # cell containing (i, j, k), i.e. coordinates halved
    par = ws.octree_order(levels=ws.LEVELS - 1)
    pi, pj, pk = par % (ni // 2), (par // (ni // 2)) % (nj // 2), par // ((ni // 2) * (nj // 2))
    v = np.arange(len(o))
    assert np.array_equal(i // 2, pi[v // 8]) and np.array_equal(j // 2, pj[v // 8]) and np.array_equal(k // 2, pk[v // 8])
    # the octant bits are di + 2 dj + 4 dk
    assert np.array_equal(v % 8, (i % 2) + 2 * (j % 2) + 4 * (k % 2))


def test_layer_table_matches_the_architecture():
    L, n = ws.layers()
    names = [l.name for l in L]
    assert names == ["enc1", "enc2", "enc3", "enc4"] + [f"{t}{i}" for i in range(1, 5) for t in ("up", "mix")] + ["out"]
    assert L[3].n == ws.CH * 16 and L[4].n == 8 * ws.CH and L[-1].n == ws.OUT_PAD
    for l in L:   # every GEMM dimension is a multiple of the tensor-core K/N step
        assert l.n % 16 == 0 and l.k % 16 == 0
    assert n == sum(l.n * l.k + l.n for l in L)


def test_state_from_conservative_inverts_the_free_stream():
    blk, prm, fs = case.bump_case(17, 9, 9)
    ro = np.full(10, fs["rho"])
    u = fs["u"]
    e = prm.rgas * fs["t"] / (prm.gamma - 1.0)
    q = np.stack([ro, ro * u, 0 * ro, 0 * ro, ro * (e + 0.5 * u * u)], axis=1)
    st = ws.state_from_conservative(q, fs, prm.gamma, prm.rgas)
    assert np.allclose(st["TEMP"], fs["t"]) and np.allclose(st["U"], u)
    assert np.allclose(st["PDIFF"], 0.0, atol=1e-9 * fs["p"])
    sc = ws.freestream_scales(fs, prm.gamma, prm.rgas)
    assert np.allclose(q[0] / sc, [1, 1, 0, 0, 1])
