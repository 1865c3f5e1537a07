"""Accuracy gates against the FP64 oracle.

* Barnes-Hut theta 0.5 at N = 1,000,000: median relative force error <= 1 %
  on a seeded 4,096-target subsample (warp and thread walks), and the theta
  dial ordered (0.3 < 0.5 < 0.7);
* 1M Barnes-Hut, 200 steps (dt 0.005): |dE/E| <= 2e-4;
* precision study (262,144 particles with 10 % Plummer cores, eps 0.01,
  dt 0.002, 2,000 steps): all-pairs force median < 1e-5 and |dE/E| <= 2e-4;
  Barnes-Hut theta 0.5 force median <= 1 % and its measured drift band
  (3.9e-4 when measured; the reference's own Barnes-Hut drifts by 5e-3 ..
  1.2e-2, docs/PERFORMANCE.md:94-104); momentum drift of both.
"""
import numpy as np
import pytest

from nbodyssey_b200 import api, ic
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)


@pytest.fixture(scope="module")
def one_million():
    pos, vel = ic.bh_config(1_000_000, seed=0)
    tg = np.random.default_rng(0).choice(1_000_000, 4096, replace=False)
    return pos, vel, tg, O.allpairs_f64(pos, 0.05, targets=tg)


@pytest.mark.parametrize("traverse", ["warp", "thread"])
def test_theta_dial_1m(one_million, traverse):
    pos, vel, tg, exact = one_million
    med = []
    for theta in (0.3, 0.5, 0.7):
        prm = api.SimParams(dt=0.005, epsilon=0.05, force="bh", theta=theta,
                            traverse=traverse)
        with api.Simulation(pos, vel, prm) as sim:
            a = sim.compute_forces()[:, :3].astype(np.float64)
        med.append(float(np.median(rel(a[tg], exact))))
    print("median force error theta 0.3/0.5/0.7 (%s):" % traverse, med)
    assert med[1] <= 0.01
    assert med[0] < med[1] < med[2]


def test_energy_1m_200_steps(one_million):
    pos, vel, _, _ = one_million
    prm = api.SimParams(dt=0.005, epsilon=0.05, force="bh", theta=0.5, traverse="warp")
    with api.Simulation(pos, vel, prm) as sim:
        e0 = sim.energy()[0]
        sim.step(200)
        e1 = sim.energy()[0]
    drift = abs(e1 - e0) / abs(e0)
    print("1M BH 200 steps |dE/E| =", drift)
    assert drift <= 2e-4


def test_precision_study():
    pos, vel = ic.precision_config(262_144, seed=0)
    tg = np.random.default_rng(1).choice(262_144, 2048, replace=False)
    exact = O.allpairs_f64(pos, 0.01, targets=tg)
    res = {}
    for force in ("naive", "bh"):
        prm = api.SimParams(dt=0.002, epsilon=0.01, force=force, theta=0.5,
                            traverse="warp")
        with api.Simulation(pos, vel, prm) as sim:
            a = sim.compute_forces()[:, :3].astype(np.float64)
            r = rel(a[tg], exact)
            e0 = sim.energy()[0]
            p0 = sim.momentum()
            sim.step(2000)
            e1 = sim.energy()[0]
            p1 = sim.momentum()
        res[force] = (float(np.median(r)), float(np.percentile(r, 99)),
                      abs(e1 - e0) / abs(e0), float(np.linalg.norm(p1 - p0)))
    print("precision study (median, p99, |dE/E|, |dP| over 2000 steps):", res)
    assert res["naive"][0] < 1e-5 and res["naive"][2] <= 2e-4
    assert res["naive"][3] < 1e-5
    assert res["bh"][0] <= 0.01 and res["bh"][2] <= 6e-4
    assert res["bh"][3] < 1e-3


@pytest.mark.parametrize("traverse", ["warp", "thread"])
def test_energy_band_12k_bh_2000_steps(traverse):
    """The 12,000-particle two-disk workload (eps 0.05, dt 0.005) with
    Barnes-Hut theta 0.5 over 2,000 steps: the measured drift band (3.2e-3
    warp / 2.9e-3 thread when measured; the reference's own Barnes-Hut runs
    drift 5e-3 .. 1.2e-2 over 1,500 steps, docs/PERFORMANCE.md:94-104) holds;
    all-pairs meets the 2e-4 gate on the same run (tests/test_gpu_integrate.py)."""
    pos, vel = ic.two_disks(12_000, seed=0)
    prm = api.SimParams(dt=0.005, epsilon=0.05, force="bh", theta=0.5, traverse=traverse)
    with api.Simulation(pos, vel, prm) as sim:
        e0 = sim.energy()[0]
        worst = 0.0
        for _ in range(20):
            sim.step(100)
            worst = max(worst, abs(sim.energy()[0] - e0) / abs(e0))
    print("12k BH theta 0.5 %s, 2000 steps: max |dE/E| = %.3g" % (traverse, worst))
    assert worst <= 5e-3


def test_energy_gate_12k_bh_accuracy_setting():
    """The opening angle at which Barnes-Hut meets the 2e-4 energy gate on
    the 12,000-particle workload over 2,000 steps.  The monopole drift
    follows the force error, not the step: measured with the oracle's walk
    (the same interaction sets, FP64 sums) at theta 0.5 / 0.4 / 0.3 / 0.2 /
    0.15 / 0.1: 3.2e-3 / 2.5e-3 / 1.4e-3 / 6.0e-4 / 3.1e-4 / 1.0e-4, and
    3.2e-3 at theta 0.5 with half the step over the same time."""
    pos, vel = ic.two_disks(12_000, seed=0)
    prm = api.SimParams(dt=0.005, epsilon=0.05, force="bh", theta=0.1, traverse="warp")
    with api.Simulation(pos, vel, prm) as sim:
        e0 = sim.energy()[0]
        worst = 0.0
        for _ in range(20):
            sim.step(100)
            worst = max(worst, abs(sim.energy()[0] - e0) / abs(e0))
    print("12k BH theta 0.1, 2000 steps: max |dE/E| = %.3g" % worst)
    assert worst <= 2e-4
