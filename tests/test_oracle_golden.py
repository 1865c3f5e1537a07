"""Pins the CPU oracle against fixtures produced by the reference's own
scripts (tests/golden/make_golden.py): lbvh_check.py's mirror of the GPU tree,
reference_nbody.py's integrator and barnes_hut_reference.py's octree."""
import os

import numpy as np
import pytest

from oracle import oracle as O


@pytest.fixture(scope="module")
def lbvh(golden_dir):
    g = np.load(os.path.join(golden_dir, "lbvh_seed1.npz"))
    n = g["pos"].shape[0]
    p4 = np.zeros((n, 4), np.float32)
    p4[:, :3] = g["pos"]
    p4[:, 3] = g["mass"]
    return g, p4


@pytest.mark.parametrize("bits", [63, 30])
def test_keys_order_topology_bit_exact(lbvh, bits):
    g, p4 = lbvh
    t = O.Tree(p4, bits)
    assert np.array_equal(t.keys, g["keys%d" % bits])
    assert np.array_equal(t.perm.astype(np.int64), g["order%d" % bits])
    assert np.array_equal(t.children, g["children%d" % bits])
    assert np.array_equal(t.parent, g["parent%d" % bits])


def test_30bit_keys_are_top_bits_of_63bit(lbvh):
    _, p4 = lbvh
    k63 = O.morton_keys(p4, 63)
    k30 = O.morton_keys(p4, 30)
    assert np.array_equal(k30, k63 >> np.uint64(33))


def test_duplicate_keys_present(lbvh):
    g, _ = lbvh
    k = g["keys63"]
    assert k.shape[0] - np.unique(k).shape[0] >= 23   # lbvh_check.py:239


def test_com_and_size(lbvh):
    g, p4 = lbvh
    t = O.Tree(p4, 63)
    # float-rounded node values against the mirror's FP64 ones
    np.testing.assert_allclose(t.com[:, :3], g["com"][:, :3], rtol=0, atol=2e-7)
    np.testing.assert_allclose(t.com[:, 3], g["com"][:, 3], rtol=2e-7)
    np.testing.assert_allclose(np.sqrt(t.size2.astype(np.float64)), g["size"],
                               rtol=1e-6, atol=1e-7)
    assert abs(t.sums[0, 3] - p4[:, 3].astype(np.float64).sum()) < 1e-9


@pytest.mark.parametrize("tag,theta", [("t00", 0.0), ("t05", 0.5)])
def test_thread_walk(lbvh, tag, theta):
    g, p4 = lbvh
    t = O.Tree(p4, 63)
    acc, inter, depth = t.walk_thread(theta, 0.05, 1.0, g["sample"])
    ref = g["thread_acc_" + tag]
    assert np.array_equal(inter, g["thread_inter_" + tag])
    assert np.array_equal(depth, g["thread_depth_" + tag])
    rel = np.linalg.norm(acc - ref, axis=1) / np.linalg.norm(ref, axis=1)
    assert rel.max() < 1e-6
    if theta == 0.0:
        assert (inter == p4.shape[0]).all()            # lbvh_check.py:260
        ex = np.linalg.norm(acc - g["exact"], axis=1) / np.linalg.norm(
            g["exact"], axis=1)
        assert ex.max() < 1e-12                        # lbvh_check.py:262
    else:
        ex = np.linalg.norm(acc - g["exact"], axis=1) / np.linalg.norm(
            g["exact"], axis=1)
        assert np.median(ex) < 0.05                    # lbvh_check.py:275
        assert inter.mean() < 0.5 * p4.shape[0]        # lbvh_check.py:276
    assert depth.max() < 128                           # lbvh_check.py:281


@pytest.mark.parametrize("tag,theta", [("t00", 0.0), ("t05", 0.5)])
def test_warp_walk(lbvh, tag, theta):
    g, p4 = lbvh
    t = O.Tree(p4, 63)
    acc, inter, depth = t.walk_warp(theta, 0.05, 1.0, g["warp_ids"])
    ref = g["warp_acc_" + tag].reshape(-1, 3)
    assert np.array_equal(inter, g["warp_inter_" + tag])
    rel = np.linalg.norm(acc - ref, axis=1) / np.linalg.norm(ref, axis=1)
    assert rel.max() < 1e-6
    if theta == 0.0:
        assert (inter == p4.shape[0]).all()


def test_warp_amplification(lbvh):
    """The warp walk does more interactions per lane than the thread walk
    (about 1.9x, docs/PERFORMANCE.md:52-53)."""
    g, p4 = lbvh
    t = O.Tree(p4, 63)
    _, it, _ = t.walk_thread(0.5, 0.05)
    _, iw, _ = t.walk_warp(0.5, 0.05)
    amp = iw.mean() / it.mean()
    assert 1.3 < amp < 3.0


def test_allpairs_against_reference_nbody(golden_dir):
    g = np.load(os.path.join(golden_dir, "refnbody.npz"))
    p4 = g["pos4"]
    a64 = O.allpairs_f64(p4, 0.05)
    np.testing.assert_allclose(a64, g["acc_f64"], rtol=1e-10, atol=1e-12)
    a32 = O.accelerations(p4[:, :3], p4[:, 3], np.float32(0.05 * 0.05),
                          np.float32(1.0), 2048, np.float32)
    assert np.array_equal(a32, g["acc_f32"])
    e = O.energy_f64(p4, g["vel4"], 0.05)
    np.testing.assert_allclose(e[:3], g["energy0"], rtol=1e-12)


@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_reference_loop_bit_exact(golden_dir, dtype):
    """The restated run loop reproduces reference_nbody.py's frames bit for
    bit and its energy rows to the printed digits."""
    from nbodyssey_b200 import formats
    g = np.load(os.path.join(golden_dir, "refnbody.npz"))
    dt = np.float32 if dtype == "float32" else np.float64
    frames, rows = O.reference_loop(g["pos4"], g["vel4"], 20, 0.01, 0.05, 1.0,
                                    5, dt)
    gold = g["frames_" + dtype]
    assert len(frames) == gold.shape[0]
    for k, fr in enumerate(frames):
        assert formats.frame_bytes(fr) == gold[k].tobytes()
    text = formats.ENERGY_HEADER + "".join(
        formats.energy_row_py(*r) for r in rows)
    assert text.encode() == g["csv_" + dtype].tobytes()


def test_octree_statistics(golden_dir):
    """The LBVH thread walk's theta error is of the octree oracle's order
    (the LBVH uses the tight-box longest edge, a conservative size)."""
    g = np.load(os.path.join(golden_dir, "bh_octree.npz"))
    p4 = g["pos4"].astype(np.float32)
    t = O.Tree(p4, 30)
    rng = np.random.default_rng(5)
    tg = rng.choice(p4.shape[0], 200, replace=False)
    ex = O.allpairs_f64(p4, 0.05, targets=tg)
    acc, inter = t.forces(0.5, 0.05)
    rel = np.linalg.norm(acc[tg] - ex, axis=1) / np.linalg.norm(ex, axis=1)
    med_oct = g["med_err"][list(g["thetas"]).index(0.5)]
    assert np.median(rel) < 3 * med_oct
    assert np.median(rel) < 0.05                       # lbvh_check.py:275
    acc0, inter0 = t.forces(0.0, 0.05)
    rel0 = np.linalg.norm(acc0[tg] - ex, axis=1) / np.linalg.norm(ex, axis=1)
    assert rel0.max() < 1e-10 and (inter0 == p4.shape[0]).all()
