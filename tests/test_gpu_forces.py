"""GPU parity of the force modules.

* Barnes-Hut walks: the interaction set of every target equals the oracle's
  (counts bit-exact, thread and warp walks); forces within 5e-5 relative of
  the oracle's FP64 sum over the same set (FP32 pair math with an
  approximate rsqrt accumulates ~1e-6).
* theta = 0 reproduces all-pairs: every target touches n leaves; forces within
  the FP32 band of the FP64 exact force; the gpu_bench.sh gate
  (mean relative difference naive vs BH < 1e-4, scripts/gpu_bench.sh:37-45).
* All-pairs: median / 99th-percentile relative error vs FP64 exact below
  2e-6 / 2e-5.
"""
import numpy as np
import pytest

from nbodyssey_b200 import api, ic
from oracle import oracle as O

pytestmark = pytest.mark.gpu

EPS = 0.05


def rel_err(a, b):
    return np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)


def assert_walk_close(acc, ref):
    """Same interaction set, FP32 sum (approximate rsqrt, ~10^3 terms in the
    walk's order) against the FP64 sum: median < 1e-6, max < 5e-5."""
    r = rel_err(acc, ref)
    assert np.median(r) < 1e-6
    assert r.max() < 5e-5


def bh_forces(pos, theta, traverse, bits=30, eps=EPS, walk="pair"):
    prm = api.SimParams(epsilon=eps, theta=theta, force="bh", traverse=traverse,
                        key_bits=bits, walk_kernel=walk)
    with api.Simulation(pos, np.zeros_like(pos), prm) as sim:
        acc, cnt = sim.debug_forces()
    return acc[:, :3].astype(np.float64), cnt.astype(np.int64)


@pytest.mark.parametrize("walk", ["pair", "list", "dfs"])
@pytest.mark.parametrize("traverse", ["thread", "warp"])
@pytest.mark.parametrize("theta", [0.3, 0.5, 0.7])
@pytest.mark.parametrize("n", [1000, 20_000, 20_001])
def test_walk_matches_oracle(n, theta, traverse, walk):
    pos, _ = ic.two_disks(n, seed=11)
    acc, cnt = bh_forces(pos, theta, traverse, walk=walk)
    ref, inter = O.Tree(pos, 30).forces(theta, EPS, traverse=traverse)
    assert np.array_equal(cnt, inter)
    assert_walk_close(acc, ref)


@pytest.mark.parametrize("walk", ["pair", "list", "dfs"])
@pytest.mark.parametrize("traverse", ["thread", "warp"])
def test_walk_matches_oracle_63bit(traverse, walk):
    pos, _ = ic.two_disks(30_000, seed=12)
    acc, cnt = bh_forces(pos, 0.5, traverse, bits=63, walk=walk)
    ref, inter = O.Tree(pos, 63).forces(0.5, EPS, traverse=traverse)
    assert np.array_equal(cnt, inter)
    assert_walk_close(acc, ref)


@pytest.mark.parametrize("walk", ["pair", "list", "dfs"])
def test_walk_1m_subsample(walk):
    """1M particles, theta 0.5 warp walk: counts of every target equal the
    oracle's (which walks only 4096 sampled warps)."""
    pos, _ = ic.bh_config(1_000_000, seed=5)
    acc, cnt = bh_forces(pos, 0.5, "warp", walk=walk)
    tree = O.Tree(pos, 30)
    rng = np.random.default_rng(0)
    warps = np.sort(rng.choice((1_000_000 + 31) // 32, 4096, replace=False))
    ref_w, inter_w, _ = tree.walk_warp(0.5, EPS, 1.0, warps)
    sorted_idx = (warps[:, None] * 32 + np.arange(32)[None, :]).ravel()
    live = sorted_idx < 1_000_000
    orig = tree.perm.astype(np.int64)[sorted_idx[live]]
    assert np.array_equal(cnt[orig], np.repeat(inter_w, 32)[live])
    assert_walk_close(acc[orig], ref_w[live])


@pytest.mark.parametrize("walk", ["pair", "list", "dfs"])
@pytest.mark.parametrize("traverse", ["thread", "warp"])
def test_theta0_equals_allpairs(traverse, walk):
    n = 20_000
    pos, _ = ic.two_disks(n, seed=13)
    acc, cnt = bh_forces(pos, 0.0, traverse, walk=walk)
    assert (cnt == n).all()
    exact = O.allpairs_f64(pos, EPS)
    r = rel_err(acc, exact)
    # FP32 accumulation of n terms in tree order; the reference's own gate is
    # a mean below 1e-4 (scripts/gpu_bench.sh:43; it published mean 1.7e-5,
    # max 2.8e-4 at 20k, docs/PERFORMANCE.md:14-20).  Near-cancelling net
    # forces set the tail.
    assert r.mean() < 1e-4
    assert np.median(r) < 1e-5 and np.percentile(r, 99) < 1e-3


def test_compare_forces_gate():
    """gpu_bench.sh's gate on --compare-forces at theta 0 (mean < 1e-4), at the
    N = 100,000 of the 1M workload's exactness gate."""
    pos, vel = ic.two_disks(100_000, seed=14)
    for tv in ("thread", "warp"):
        prm = api.SimParams(epsilon=EPS, theta=0.0, force="bh", traverse=tv)
        with api.Simulation(pos, vel, prm) as sim:
            mx, mean = sim.compare_forces()
        assert mean < 1e-4 and mx < 1e-3


@pytest.mark.parametrize("traverse", ["thread", "warp"])
def test_theta0_100k_equals_fp64_allpairs(traverse):
    """The theta = 0 exactness gate at N = 100,000: every target touches all
    n leaves, and the forces of a seeded 2,048-target subsample are within
    the FP32 all-pairs band of the FP64 exact force."""
    n = 100_000
    pos, _ = ic.two_disks(n, seed=15)
    acc, cnt = bh_forces(pos, 0.0, traverse)
    assert (cnt == n).all()
    tg = np.random.default_rng(15).choice(n, 2048, replace=False)
    r = rel_err(acc[tg], O.allpairs_f64(pos, EPS, targets=tg))
    # the reference's gate (mean < 1e-4, scripts/gpu_bench.sh:43); FP32
    # accumulation of 1e5 terms in tree order puts the median near 1e-5
    # (1.0e-5 measured), about sqrt(5) above the 20k case's
    assert r.mean() < 1e-4
    assert np.median(r) < 3e-5 and np.percentile(r, 99) < 1e-3


@pytest.mark.parametrize("n", [1, 2, 3, 33, 511, 512, 513, 4096, 12_000, 50_001])
def test_allpairs_vs_fp64(n):
    pos, _ = ic.two_disks(max(n, 2), seed=n)
    pos = pos[:n]
    prm = api.SimParams(epsilon=EPS, force="naive")
    with api.Simulation(pos, np.zeros_like(pos), prm) as sim:
        acc = sim.compute_forces()
    assert np.all(acc[:, 3] == 0.0)
    exact = O.allpairs_f64(pos, EPS)
    if n == 1:
        assert np.all(acc[:, :3] == 0.0)
        return
    r = rel_err(acc[:, :3].astype(np.float64), exact)
    assert np.median(r) < 2e-6
    assert np.percentile(r, 99) < 2e-5


def test_allpairs_reference_golden(golden_dir):
    """The reference's own FP64 accelerations of its fixture IC."""
    import os
    g = np.load(os.path.join(golden_dir, "refnbody.npz"))
    prm = api.SimParams(epsilon=EPS, force="naive")
    with api.Simulation(g["pos4"], g["vel4"], prm) as sim:
        acc = sim.compute_forces()[:, :3].astype(np.float64)
    r = rel_err(acc, g["acc_f64"])
    assert np.percentile(r, 99) < 2e-5


def test_bh_small_n_edge_cases():
    # n = 1: the reference writes zeros (src/forces_bh.cu:466-469)
    p1 = np.array([[0.5, 0.5, 0.5, 1.0]], np.float32)
    acc, _ = bh_forces(p1, 0.5, "warp")
    assert np.all(acc == 0.0)
    p2 = np.array([[0, 0, 0, 1.0], [1, 0, 0, 1.0]], np.float32)
    acc, cnt = bh_forces(p2, 0.5, "thread")
    ex = O.allpairs_f64(p2, EPS)
    assert rel_err(acc, ex).max() < 1e-5


def test_theta05_accuracy_vs_fp64():
    """theta 0.5: median and 99th-percentile force error vs FP64, the dial
    of docs/PERFORMANCE.md:84-88 (reported; the LBVH's tight-box size makes
    it at least as accurate as the octree at the same theta)."""
    pos, _ = ic.two_disks(100_000, seed=15)
    rng = np.random.default_rng(1)
    tg = rng.choice(100_000, 2048, replace=False)
    exact = O.allpairs_f64(pos, EPS, targets=tg)
    for tv in ("thread", "warp"):
        acc, _ = bh_forces(pos, 0.5, tv)
        r = rel_err(acc[tg], exact)
        assert np.median(r) < 0.05                     # lbvh_check.py:275
        if tv == "warp":
            assert np.median(r) < 0.02


@pytest.mark.parametrize("n,expect", [(5_000, "naive"), (30_000, "bh")])
def test_auto_force_picks_by_crossover(n, expect):
    """force=auto is the all-pairs module below 20,000 particles and
    Barnes-Hut from there on, bit for bit."""
    pos, vel = ic.two_disks(n, seed=18)
    out = {}
    for force in ("auto", expect):
        prm = api.SimParams(dt=0.005, epsilon=EPS, theta=0.5, force=force,
                            traverse="warp")
        with api.Simulation(pos, vel, prm) as sim:
            sim.step(2)
            out[force] = (sim.positions(), sim.velocities())
    assert np.array_equal(out["auto"][0], out[expect][0])
    assert np.array_equal(out["auto"][1], out[expect][1])


def test_determinism():
    pos, _ = ic.two_disks(50_000, seed=16)
    a1, _ = bh_forces(pos, 0.5, "warp")
    a2, _ = bh_forces(pos, 0.5, "warp")
    assert np.array_equal(a1, a2)
    prm = api.SimParams(epsilon=EPS, force="naive")
    with api.Simulation(pos, np.zeros_like(pos), prm) as sim:
        b1 = sim.compute_forces()
        b2 = sim.compute_forces()
    assert np.array_equal(b1, b2)


@pytest.mark.parametrize("traverse", ["thread", "warp"])
def test_list_walk_duplicates_and_clumps(traverse):
    """Coincident clumps (zero-size nodes, duplicate keys) through the list
    walk's box prefilter: interaction sets still equal the oracle's."""
    rng = np.random.default_rng(9)
    p = np.zeros((6000, 4), np.float32)
    p[:, :3] = rng.normal(size=(6000, 3)).astype(np.float32)
    p[:1500, :3] = np.float32([0.25, -0.5, 0.75])
    p[1500:1800, :3] = p[1600, :3]
    p[:, 3] = 1.0 / 6000
    for theta in (0.0, 0.5, 1.0):
        acc, cnt = bh_forces(p, theta, traverse)
        ref, inter = O.Tree(p, 30).forces(theta, EPS, traverse=traverse)
        assert np.array_equal(cnt, inter)
        if theta == 0.0:   # all 6000 terms: the theta = 0 band
            r = rel_err(acc, ref)
            assert r.mean() < 1e-4 and np.median(r) < 1e-5
        else:
            assert_walk_close(acc, ref)


@pytest.mark.parametrize("walk", ["pair", "list"])
def test_batched_and_dfs_thread_walks_agree(walk):
    """The lane-masked batched walks give every target its per-thread
    interaction set: counts equal the one-thread-per-target walk's."""
    pos, _ = ic.two_disks(50_000, seed=17)
    a1, c1 = bh_forces(pos, 0.5, "thread", walk=walk)
    a2, c2 = bh_forces(pos, 0.5, "thread", walk="dfs")
    assert np.array_equal(c1, c2)
    assert_walk_close(a1, a2.astype(np.float64))
