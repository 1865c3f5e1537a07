"""Serving with continuous batching: requests that arrive while others run are
admitted as slots free up, run together on the device, and each result is
bit-identical to the same request run alone through the handle API.
Frames stream out in the reference layout; sizes beyond the budget are
refused."""
import dataclasses
import os
import threading
import time

import numpy as np
import pytest

from nbodyssey_b200 import _lib as L
from nbodyssey_b200 import api, formats, ic
from nbodyssey_b200.server import DONE, Server

pytestmark = pytest.mark.gpu


def _request(k, forces=("bh",)):
    n = (3000, 40, 17_000, 2, 9000, 1)[k % 6]
    if n == 1:
        p = np.array([[0.25, 0.5, -0.5, 0.3]], np.float32)
        pos, vel = p, np.full_like(p, 0.01)
    else:
        pos, vel = ic.two_disks(max(n, 2), seed=200 + k, impact=2.0 + k % 5)
        pos, vel = pos[:n], vel[:n]
    prm = api.SimParams(dt=0.005, epsilon=0.05, force=forces[k % len(forces)],
                        theta=(0.3, 0.5, 0.7)[k % 3],
                        traverse=("warp", "thread")[k % 2])
    steps = (7, 3, 12, 5, 9, 4)[k % 6]
    return pos, vel, prm, steps


def _alone(pos, vel, prm, steps):
    with api.Simulation(pos, vel, prm) as sim:
        sim.step(steps)
        return sim.positions(), sim.velocities()


def test_results_identical_alone_and_in_the_mix(tmp_path):
    reqs = [_request(k) for k in range(12)]
    # a small pool: not every request fits at once, so admission waits for
    # running ones to finish (continuous batching, not a fixed batch)
    with Server(hbm_budget_bytes=16 << 20, max_sims=8) as srv:
        ids = []
        for k, (pos, vel, prm, steps) in enumerate(reqs):
            ids.append(srv.submit(pos, vel, prm, steps,
                                  dump_every=2 if k == 0 else 0,
                                  out_dir=str(tmp_path / "f0") if k == 0 else None))
            if k % 4 == 3:
                time.sleep(0.01)   # later requests arrive while others run
        for rid in ids:
            srv.wait(rid, 120)
        polls = [srv.poll(rid) for rid in ids]
        results = [srv.result(rid) for rid in ids]
        st = srv.stats()
    assert all(p[0] == DONE for p in polls)
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["peak_running"] >= 2
    for (pos, vel, prm, steps), (p, v) in zip(reqs, results):
        ap, av = _alone(pos, vel, prm, steps)
        assert np.array_equal(p, ap)
        assert np.array_equal(v, av)
    # frames of request 0: steps 0, 2, 4, 6 of 7
    names = sorted(os.listdir(tmp_path / "f0"))
    assert names == ["frame_%05d.bin" % k for k in range(4)]
    assert formats.read_frame(str(tmp_path / "f0" / names[0])).shape == reqs[0][0].shape


def test_all_pairs_and_auto_requests_identical_alone():
    """All-pairs requests (the persistent work-queue launch, scratch from the
    all-pairs pool), AUTO and Barnes-Hut requests in one stream: each result
    equals the request run alone."""
    reqs = [_request(k, ("naive", "auto", "bh", "naive")) for k in range(12)]
    with Server(hbm_budget_bytes=256 << 20, max_sims=6) as srv:
        ids = []
        for k, (pos, vel, prm, steps) in enumerate(reqs):
            ids.append(srv.submit(pos, vel, prm, steps))
            if k % 3 == 2:
                time.sleep(0.01)
        for rid in ids:
            srv.wait(rid, 120)
        used = [srv.force(rid) for rid in ids]
        results = [srv.result(rid) for rid in ids]
        st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert "naive" in used and "bh" in used
    for (pos, vel, prm, steps), (p, v), f in zip(reqs, results, used):
        # AUTO resolves by the batch crossover: alone, the same module
        ap, av = _alone(pos, vel, dataclasses.replace(prm, force=f), steps)
        assert np.array_equal(p, ap)
        assert np.array_equal(v, av)


def test_concurrent_submitters():
    reqs = [_request(k) for k in range(8)]
    out = {}
    with Server(hbm_budget_bytes=64 << 20, max_sims=16) as srv:
        def client(k):
            pos, vel, prm, steps = reqs[k]
            rid = srv.submit(pos, vel, prm, steps)
            srv.wait(rid, 120)
            out[k] = srv.result(rid)
        th = [threading.Thread(target=client, args=(k,)) for k in range(len(reqs))]
        for t in th:
            t.start()
        for t in th:
            t.join()
    for k, (pos, vel, prm, steps) in enumerate(reqs):
        ap, av = _alone(pos, vel, prm, steps)
        assert np.array_equal(out[k][0], ap) and np.array_equal(out[k][1], av)


def test_refuses_what_cannot_fit_and_bad_params():
    with Server(hbm_budget_bytes=16 << 20, max_sims=4) as srv:
        big = np.zeros((200_000, 4), np.float32)
        with pytest.raises(L.NbError) as ei:
            srv.submit(big, big, api.SimParams(force="bh"), 1)
        assert ei.value.code == L.NB_ERR_NOMEM
        small, _ = ic.two_disks(100, seed=3)
        with pytest.raises(L.NbError) as ei:
            srv.submit(small, small, api.SimParams(force="bh", key_bits=63), 1)
        assert ei.value.code == L.NB_ERR_INVALID
        # an all-pairs request whose scratch exceeds the all-pairs pool
        mid, _ = ic.two_disks(30_000, seed=4)
        with pytest.raises(L.NbError) as ei:
            srv.submit(mid, mid, api.SimParams(force="naive"), 1)
        assert ei.value.code == L.NB_ERR_NOMEM
        with pytest.raises(L.NbError) as ei:
            srv.result(12345)
        assert ei.value.code == L.NB_ERR_NOTFOUND
