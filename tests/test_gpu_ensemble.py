"""GPU parity of batched ensembles: every simulation of an ensemble ends in
exactly the state (bit for bit) it reaches when run alone through the handle
API with the same parameters, whatever else is in the mix; energies too."""
import dataclasses

import numpy as np
import pytest

from nbodyssey_b200 import _lib as L
from nbodyssey_b200 import api, ic
from nbodyssey_b200.ensemble import Ensemble

pytestmark = pytest.mark.gpu


def _mix(forces=("bh",)):
    sizes = [1, 2, 33, 1000, 4097, 20_000, 64, 3000]
    states, params = [], []
    for k, n in enumerate(sizes):
        states.append(ic.two_disks(max(n, 2), seed=100 + k, mass_ratio=0.5 + 0.05 * k,
                                   impact=2.0 + k)
                      if n > 1 else None)
        if n == 1:
            p = np.array([[0.5, -0.25, 0.125, 1.0]], np.float32)
            states[-1] = (p, np.zeros_like(p))
        else:
            states[-1] = (states[-1][0][:n], states[-1][1][:n])
        params.append(api.SimParams(dt=0.005, epsilon=0.05, force=forces[k % len(forces)],
                                    theta=(0.3, 0.5, 0.7)[k % 3],
                                    traverse=("warp", "thread")[k % 2]))
    return states, params


@pytest.mark.parametrize("forces", [("bh",), ("naive", "auto", "bh"), ("naive",)])
def test_ensemble_equals_alone(forces):
    """Barnes-Hut, all-pairs (the persistent work-queue launch) and
    NB_FORCE_AUTO simulations side by side: each equals itself alone."""
    states, params = _mix(forces)
    steps = 4
    with Ensemble(states, params) as ens:
        ens.step(steps)
        ens.sync()
        got = [ens.state(s) for s in range(ens.nsims)]
        acc = [ens.accelerations(s) for s in range(ens.nsims)]
        e_ens = ens.energy()
        # AUTO resolves by the batch crossover: alone, the same module
        forces_used = [ens.force(s) for s in range(ens.nsims)]
    for s, ((pos, vel), prm) in enumerate(zip(states, params)):
        prm = dataclasses.replace(prm, force=forces_used[s])
        with api.Simulation(pos, vel, prm) as sim:
            sim.step(steps)
            p, v, a = sim.positions(), sim.velocities(), sim.compute_forces()
            e = sim.energy()
        assert np.array_equal(got[s][0], p), s
        assert np.array_equal(got[s][1], v), s
        assert np.array_equal(acc[s], a), s
        assert np.array_equal(e_ens[s], np.array(e)), s


def test_ensemble_graph_and_eager_identical():
    states, params = _mix(("naive", "bh"))
    out = []
    for graphs in (True, False):
        with Ensemble(states, params) as ens:
            ens.set_graphs(graphs)
            ens.step(3)
            out.append([ens.state(s)[0] for s in range(ens.nsims)])
    for a, b in zip(*out):
        assert np.array_equal(a, b)


def test_ensemble_rejects_unsupported_params():
    pos, vel = ic.two_disks(100, seed=1)
    with pytest.raises(L.NbError) as ei:
        Ensemble([(pos, vel)], api.SimParams(force="bh", key_bits=63))
    assert ei.value.code == L.NB_ERR_INVALID
    with pytest.raises(L.NbError):
        Ensemble([(pos, vel)], api.SimParams(force="bh", epsilon=0.0))


def test_ensemble_kernels_per_step():
    """The launch count a step reports: prep, then the tree pipeline (Morton
    keys, five sort passes, the build levels, one walk launch per semantics
    in use) when some simulation uses Barnes-Hut, and the all-pairs packing
    plus one queue launch per launch shape when some uses all-pairs."""
    states, params = _mix(("bh",))
    warp_only = [dataclasses.replace(p, traverse="warp") for p in params]
    with Ensemble(states, warp_only) as ens:
        k_warp = ens.kernels_per_step()
    with Ensemble(states, params) as ens:
        k_both = ens.kernels_per_step()
    assert k_both == k_warp + 1                 # a second walk launch
    assert k_warp >= 1 + 1 + 5 + 1 + 1          # prep, Morton, sort, >= 1 level, walk
    states, params = _mix(("naive",))
    with Ensemble(states, params) as ens:
        k_ap = ens.kernels_per_step()
    assert 3 <= k_ap <= 1 + 1 + 6               # prep, pack, 1..6 queue shapes
