"""A Barnes-Hut simulation split over ranks (nb_forces_range_dev +
nb_forces_gather_dev, nbodyssey_b200/shard.py), on one GPU: R ranks are
emulated by R engines with their own state and workspace, and the exchange
by concatenating their parts.  Every rank's state must equal the one-GPU
simulation's bit for bit after several steps (same tree, same interaction
sets, same float operations)."""
import ctypes

import numpy as np
import pytest

from nbodyssey_b200 import _lib as L
from nbodyssey_b200 import api, ic
from nbodyssey_b200.shard import NativeEngine, ShardedSimulation, shard_range

pytestmark = pytest.mark.gpu


def _reference(pos, vel, prm, steps):
    with api.Simulation(pos, vel, prm) as sim:
        sim.compute_forces()
        sim.step(steps)
        return sim.positions(), sim.velocities(), sim.compute_forces()


def _emulated(pos, vel, prm, world, steps):
    torch = pytest.importorskip("torch")
    n = pos.shape[0]
    engines = [NativeEngine(pos, vel, prm) for _ in range(world)]
    ranges = [shard_range(n, r, world) for r in range(world)]
    chunk = ranges[0][2]
    parts = [e.alloc(chunk) for e in engines]
    try:
        for s in range(steps + 1):
            kick = s > 0   # the first pass is a(x) before the loop
            for e, (t0, t1, _), part in zip(engines, ranges, parts):
                e.forces_range(t0, t1, part, kick)
            gathered = torch.cat(parts)   # the all-gather
            for e in engines:
                e.gather(gathered.to(e.pos.device), kick)
        return [e.state() for e in engines]
    finally:
        for e in engines:
            e.close()


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_split_walk_bit_identical(world):
    pos, vel = ic.two_disks(20_001, seed=41)
    prm = api.SimParams(dt=0.005, epsilon=0.05, theta=0.5, force="bh",
                        traverse="warp")
    ref = _reference(pos, vel, prm, 3)
    for st in _emulated(pos, vel, prm, world, 3):
        for got, want in zip(st, ref):
            assert np.array_equal(got, want)


@pytest.mark.parametrize("traverse,bits", [("thread", 30), ("warp", 63)])
def test_split_walk_other_modes(traverse, bits):
    pos, vel = ic.two_disks(9_000, seed=42)
    prm = api.SimParams(dt=0.005, epsilon=0.05, theta=0.7, force="bh",
                        traverse=traverse, key_bits=bits)
    ref = _reference(pos, vel, prm, 2)
    for st in _emulated(pos, vel, prm, 4, 2):
        for got, want in zip(st, ref):
            assert np.array_equal(got, want)


def test_one_rank_sharded_simulation_equals_simulation():
    pos, vel = ic.two_disks(12_345, seed=43)
    prm = api.SimParams(dt=0.005, epsilon=0.05, theta=0.5, force="bh",
                        traverse="warp")
    ref = _reference(pos, vel, prm, 4)
    with ShardedSimulation(pos, vel, prm) as sim:
        sim.step(4)
        p, v, a = sim.state()
    assert np.array_equal(p, ref[0]) and np.array_equal(v, ref[1])
    assert np.array_equal(a, ref[2])


def test_range_arguments_checked():
    torch = pytest.importorskip("torch")
    pos, vel = ic.two_disks(1000, seed=44)
    prm = api.SimParams(epsilon=0.05, force="bh", traverse="warp")
    e = NativeEngine(pos, vel, prm)
    part = e.alloc(1000)
    try:
        for t0, t1 in ((5, 64), (0, 33), (64, 32), (0, 1001), (-32, 0)):
            with pytest.raises(L.NbError):
                e.forces_range(t0, t1, part, False)
        e.forces_range(0, 1000, part, False)   # t1 = n need not be aligned
        naive = NativeEngine(pos, vel, api.SimParams(epsilon=0.05, force="naive"))
        try:
            with pytest.raises(L.NbError):
                naive.forces_range(0, 1000, naive.alloc(1000), False)
        finally:
            naive.close()
        torch.cuda.synchronize()
    finally:
        e.close()


def test_tiny_and_empty_ranges():
    """n = 1 (no tree: zero force) and ranks whose range is empty."""
    pos = np.array([[0.1, 0.2, 0.3, 1.0]], np.float32)
    vel = np.array([[1.0, 0.0, 0.0, 0.0]], np.float32)
    prm = api.SimParams(dt=0.01, epsilon=0.05, force="bh", traverse="warp")
    ref = _reference(pos, vel, prm, 2)
    for st in _emulated(pos, vel, prm, 3, 2):
        for got, want in zip(st, ref):
            assert np.array_equal(got, want)
    pos, vel = ic.two_disks(40, seed=45)   # 2 warps over 4 ranks
    ref = _reference(pos, vel, prm, 2)
    for st in _emulated(pos, vel, prm, 4, 2):
        for got, want in zip(st, ref):
            assert np.array_equal(got, want)
