"""GPU parity of the LBVH build against the CPU oracle: Morton keys, the
sort permutation, the Karras topology, centres of mass and sizes are
bit-exact (the oracle mirrors the device's float operations); the oracle is
itself pinned to scripts/lbvh_check.py (tests/test_oracle_golden.py)."""
import os

import numpy as np
import pytest

from nbodyssey_b200 import api, ic
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _lbvh_fixture(golden_dir):
    g = np.load(os.path.join(golden_dir, "lbvh_seed1.npz"))
    n = g["pos"].shape[0]
    p4 = np.zeros((n, 4), np.float32)
    p4[:, :3] = g["pos"]
    p4[:, 3] = g["mass"]
    return g, p4


def _device_tree(p4, bits, traverse="warp"):
    prm = api.SimParams(epsilon=0.05, theta=0.5, force="bh", traverse=traverse,
                        key_bits=bits)
    with api.Simulation(p4, np.zeros_like(p4), prm) as sim:
        return sim.debug_lbvh()


def _assert_tree_equal(t, o, bits):
    k = o.keys_sorted if bits == 63 else o.keys_sorted
    assert np.array_equal(t["keys"], k)
    assert np.array_equal(t["perm"], o.perm)
    assert np.array_equal(t["children"], o.children)
    assert np.array_equal(t["parent"], o.parent)
    assert np.array_equal(t["com4"], o.com)
    assert np.array_equal(t["size2"], o.size2)


@pytest.mark.parametrize("bits", [30, 63])
def test_reference_fixture_bit_exact(golden_dir, bits):
    """lbvh_check.py's own case: keys, order and topology equal the
    reference mirror's (golden), and everything equals the oracle."""
    g, p4 = _lbvh_fixture(golden_dir)
    t = _device_tree(p4, bits)
    assert np.array_equal(t["perm"].astype(np.int64), g["order%d" % bits])
    assert np.array_equal(t["children"], g["children%d" % bits])
    assert np.array_equal(t["parent"], g["parent%d" % bits])
    gk = np.sort(g["keys%d" % bits])
    assert np.array_equal(t["keys"], gk)
    _assert_tree_equal(t, O.Tree(p4, bits), bits)


# 1023 .. 3073 straddle the 1024-leaf groups of the bottom-up build, 4095 ..
# 4097 the sort's 4096-key tiles (2047 .. 2049 half a tile)
@pytest.mark.parametrize("n", [2, 3, 31, 33, 1000, 1023, 1024, 1025, 2047, 2048, 2049,
                               3073, 4095, 4096, 4097, 100_003])
@pytest.mark.parametrize("bits", [30, 63])
def test_sizes_bit_exact(n, bits):
    pos, _ = ic.two_disks(n, seed=n)
    _assert_tree_equal(_device_tree(pos, bits), O.Tree(pos, bits), bits)


def test_duplicates_and_coincident_points():
    """Many identical keys: the index tie-break keeps a valid tree."""
    rng = np.random.default_rng(4)
    p = np.zeros((5000, 4), np.float32)
    p[:, :3] = rng.normal(size=(5000, 3)).astype(np.float32)
    p[:2000, :3] = np.float32([0.123, -0.456, 0.789])   # coincident clump
    p[2000:2600, :3] = p[2000, :3]
    p[:, 3] = 1.0 / 5000
    for bits in (30, 63):
        _assert_tree_equal(_device_tree(p, bits), O.Tree(p, bits), bits)


@pytest.mark.parametrize("n", [700, 5000])
def test_all_points_coincident(n):
    """One key for every particle: the tree is the index tie-break's alone
    (5000 spans several build groups)."""
    p = np.zeros((n, 4), np.float32)
    p[:, :3] = 1.5
    p[:, 3] = 1.0
    _assert_tree_equal(_device_tree(p, 30), O.Tree(p, 30), 30)


def test_large_tree_bit_exact_1m():
    """The Barnes-Hut workload size: 1,000,000 particles, 30-bit keys."""
    pos, _ = ic.bh_config(1_000_000, seed=3)
    t = _device_tree(pos, 30)
    o = O.Tree(pos, 30)
    _assert_tree_equal(t, o, 30)
    # size-independent properties: keys sorted, permutation is a permutation
    assert np.all(np.diff(t["keys"].astype(np.int64)) >= 0)
    assert np.array_equal(np.sort(t["perm"]), np.arange(1_000_000, dtype=np.uint32))
    assert abs(float(t["com4"][0, 3]) - float(pos[:, 3].astype(np.float64).sum())) < 1e-5


@pytest.mark.parametrize("n,bits,layout", [(4_194_305, 30, "disks"), (300_001, 63, "disks"),
                                           (300_001, 30, "coincident")])
def test_levels_above_groups_bit_exact(n, bits, layout):
    """Trees with several levels above the 1024-leaf groups (4M: four
    later launches; coincident points: the longest open-split segments)."""
    if layout == "coincident":
        pos = np.zeros((n, 4), np.float32)
        pos[:, :3] = -0.75
        pos[:, 3] = 1.0 / n
    else:
        pos, _ = ic.two_disks(n, seed=n)
    _assert_tree_equal(_device_tree(pos, bits), O.Tree(pos, bits), bits)


def expected_pairs(o):
    """The child-pair records implied by the oracle's tree: record k holds the
    children of the internal node whose split is after sorted leaf k."""
    n = o.n
    ni = n - 1
    rec = np.zeros((ni, 12), np.float32)
    for p in range(ni):
        l, r = int(o.children[p, 0]), int(o.children[p, 1])
        k = l if l < ni else l - ni   # the node's split: its left child's index
        for side, c in ((0, l), (1, r)):
            if c >= ni:   # leaf
                x, y, z, m = o.pos_sorted[c - ni]
                s2, w = np.float32(-1.0), -1
            else:
                x, y, z, m = o.com[c]
                s2 = o.size2[c]
                cl = int(o.children[c, 0])
                w = cl if cl < ni else cl - ni
            rec[k, 4 * side: 4 * side + 4] = (x, y, z, m)
            rec[k, 8 + 2 * side] = s2
            rec[k, 9 + 2 * side] = np.int32(w).view(np.float32)
    return rec


@pytest.mark.parametrize("n", [2, 3, 33, 1025, 4097, 20_001])
@pytest.mark.parametrize("bits", [30, 63])
def test_child_pair_records_bit_exact(n, bits):
    """Every child-pair record the build writes (the walk's input) equals the
    record derived from the oracle's tree, bits of the floats included."""
    pos, _ = ic.two_disks(max(n, 4), seed=n + 7)
    pos = pos[:n]
    prm = api.SimParams(epsilon=0.05, theta=0.5, force="bh", traverse="warp", key_bits=bits)
    with api.Simulation(pos, np.zeros_like(pos), prm) as sim:
        rec = sim.debug_pairs()
    exp = expected_pairs(O.Tree(pos, bits))
    assert np.array_equal(rec.view(np.int32), exp.view(np.int32))
