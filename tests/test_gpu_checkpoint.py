"""Checkpoint / resume: K steps, a state file, a new simulation from it and
K more steps give bit for bit the state of 2K uninterrupted steps (positions
with their low-order parts, velocities and a(x)); the state file's ic.bin
prefix is the state's positions and velocities (docs/FORMATS.md:8-16)."""
import numpy as np
import pytest

from nbodyssey_b200 import api, formats, ic

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("force,traverse", [("bh", "warp"), ("bh", "thread"),
                                            ("naive", "warp")])
def test_resume_is_bit_identical(tmp_path, force, traverse):
    pos, vel = ic.two_disks(20_000, seed=21)
    prm = api.SimParams(dt=0.005, epsilon=0.05, theta=0.5, force=force,
                        traverse=traverse)
    K = 25
    path = str(tmp_path / "state.bin")

    def snapshot(sim):
        return (sim.positions(), sim.position_lo(), sim.velocities(), sim.accelerations())

    with api.Simulation(pos, vel, prm) as a:
        a.step(2 * K)
        ref = snapshot(a)
    with api.Simulation(pos, vel, prm) as b:
        b.step(K)
        mid = snapshot(b)
        b.save_state(path)
    st = api.read_state(path)
    assert np.array_equal(st["pos"], mid[0]) and np.array_equal(st["lo"], mid[1])
    p_ic, v_ic = formats.read_ic(path)
    assert np.array_equal(p_ic, mid[0]) and np.array_equal(v_ic, mid[2])
    with api.Simulation.from_state(path) as c:
        assert c.params.force == force and c.params.traverse == traverse
        c.step(K)
        got = snapshot(c)
    for r, g in zip(ref, got):
        assert np.array_equal(r, g)


def test_load_state_into_existing_simulation(tmp_path):
    pos, vel = ic.two_disks(4096, seed=22)
    prm = api.SimParams(dt=0.005, epsilon=0.05, theta=0.5, force="bh", traverse="warp")
    path = str(tmp_path / "s.bin")
    with api.Simulation(pos, vel, prm) as a:
        a.step(10)
        a.save_state(path)
        a.step(10)
        ref = a.positions()
    other = api.SimParams(dt=0.01, epsilon=0.1, force="naive")
    with api.Simulation(pos, vel, other) as b:
        b.load_state(path)
        assert abs(b.params.dt - 0.005) < 1e-9 and b.params.force == "bh"
        b.step(10)
        assert np.array_equal(b.positions(), ref)
