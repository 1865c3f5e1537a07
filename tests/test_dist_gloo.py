"""Multi-process paths on CPU (gloo, world size 2): bench.py's rank plumbing
(max over ranks, barrier) and the sharding of independent simulations over
ranks, which needs no collective (each rank runs its own share)."""
import os
import socket
import subprocess
import sys

import pytest

from nbodyssey_b200.ensemble import shard

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


WORKER = r"""
import os, sys, json
sys.path.insert(0, sys.argv[1])
import bench
from nbodyssey_b200.ensemble import shard
rank, world, local, pg = bench.dist_setup()
assert pg is not None and pg.get_backend() == "gloo"
m = bench.dist_max(pg, float(rank + 1) * 1.5)
bench.dist_barrier(pg)
sizes = [2048 * (k + 1) for k in range(9)]
mine = shard(sizes, rank, world)
import torch
t = torch.zeros(len(sizes), dtype=torch.int64)
for i in mine:
    t[i] += 1
pg.all_reduce(t)
print(json.dumps({"rank": rank, "max": m, "mine": mine, "cover": t.tolist()}))
pg.destroy_process_group()
"""


def test_two_ranks_gloo(tmp_path):
    script = tmp_path / "worker.py"
    script.write_text(WORKER)
    port = _free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE="2", LOCAL_RANK=str(r),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                   CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, str(script), ROOT], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                                      text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=240)
        assert p.returncode == 0, err
        outs.append(out.strip().splitlines()[-1])
    import json
    res = sorted((json.loads(o) for o in outs), key=lambda d: d["rank"])
    assert all(d["max"] == 3.0 for d in res)              # max over ranks
    assert res[0]["cover"] == [1] * 9                       # every sim exactly once
    assert set(res[0]["mine"]).isdisjoint(res[1]["mine"])


def test_shard_balances_and_is_deterministic():
    sizes = [131072, 2048, 65536, 4096, 32768, 8192, 16384, 2048]
    a = shard(sizes, 0, 2)
    b = shard(sizes, 1, 2)
    assert sorted(a + b) == list(range(len(sizes)))
    la = sum(sizes[i] for i in a)
    lb = sum(sizes[i] for i in b)
    assert abs(la - lb) <= max(sizes)
    assert shard(sizes, 0, 2) == a
    assert shard(sizes, 0, 1) == list(range(len(sizes)))


# --- one simulation split over ranks (nbodyssey_b200/shard.py) ---------------
# The device work is replaced by a numpy engine with the same interface:
# "sorted order" is the order of x, forces are all-pairs (independent of the
# target range), kick / drift as the leapfrog.  Any split over ranks must
# then reproduce the one-rank run exactly: the test covers the ranges, the
# padded chunks, the all-gather and the step order.
FAKE_ENGINE = r"""
import numpy as np
import torch


class FakeEngine:
    def __init__(self, pos, vel, dt=0.01, eps=0.05):
        self.pos, self.vel = pos.copy(), vel.copy()
        self.acc = np.zeros_like(pos)
        self.n, self.h, self.dt, self.e2 = pos.shape[0], np.float32(dt / 2), np.float32(dt), eps * eps
        self.perm = None

    def alloc(self, rows):
        return torch.zeros((rows, 4), dtype=torch.float32)

    def _forces(self):
        p = self.pos.astype(np.float64)
        d = p[None, :, :3] - p[:, None, :3]
        r2 = (d * d).sum(-1) + self.e2
        w = p[None, :, 3] / r2 ** 1.5
        a = np.zeros_like(self.pos)
        a[:, :3] = (d * w[..., None]).sum(1)
        return a

    def forces_range(self, t0, t1, part, kick):
        if kick:
            self.vel[:, :3] += self.h * self.acc[:, :3]
            self.pos[:, :3] += self.dt * self.vel[:, :3]
        self.perm = np.argsort(self.pos[:, 0], kind="stable")
        part[: t1 - t0] = torch.from_numpy(self._forces()[self.perm[t0:t1]])

    def gather(self, sorted_all, kick):
        self.acc[self.perm] = sorted_all[: self.n].numpy()
        if kick:
            self.vel[:, :3] += self.h * self.acc[:, :3]

    def state(self):
        return self.pos.copy(), self.vel.copy(), self.acc.copy()


def initial(n):
    rng = np.random.default_rng(n)
    pos = rng.normal(size=(n, 4)).astype(np.float32)
    pos[:, 3] = 1.0 / n
    vel = (0.1 * rng.normal(size=(n, 4))).astype(np.float32)
    vel[:, 3] = 0
    return pos, vel
"""

SHARD_WORKER = r"""
import os, sys
sys.path.insert(0, sys.argv[1])
sys.path.insert(0, sys.argv[2])
import numpy as np
import bench
from fake_engine import FakeEngine, initial
from nbodyssey_b200.shard import ShardedSimulation
rank, world, local, pg = bench.dist_setup()
n = int(sys.argv[3])
pos, vel = initial(n)
sim = ShardedSimulation(pos, vel, None, engine=FakeEngine(pos, vel))
assert (sim.rank, sim.world) == (rank, world)
sim.step(3)
np.save(os.path.join(sys.argv[2], "state_%d.npy" % rank), np.stack(sim.state()))
pg.destroy_process_group()
"""


@pytest.mark.parametrize("world,n", [(2, 200), (3, 200), (4, 70)])
def test_split_simulation_ranks_gloo(tmp_path, world, n):
    """Every rank ends with the one-rank state; n = 70 over 4 ranks leaves
    the last rank an empty range."""
    import numpy as np
    (tmp_path / "fake_engine.py").write_text(FAKE_ENGINE)
    script = tmp_path / "worker.py"
    script.write_text(SHARD_WORKER)
    port = _free_port()
    procs = []
    for r in range(world):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE=str(world), LOCAL_RANK=str(r),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                   CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, str(script), ROOT, str(tmp_path),
                                       str(n)], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    for p in procs:
        out, err = p.communicate(timeout=240)
        assert p.returncode == 0, err
    sys.path.insert(0, str(tmp_path))
    try:
        from fake_engine import FakeEngine, initial
    finally:
        sys.path.remove(str(tmp_path))
    from nbodyssey_b200.shard import ShardedSimulation
    pos, vel = initial(n)
    one = ShardedSimulation(pos, vel, None, engine=FakeEngine(pos, vel))
    one.step(3)
    want = np.stack(one.state())
    for r in range(world):
        got = np.load(tmp_path / ("state_%d.npy" % r))
        assert np.array_equal(got, want)


def test_shard_ranges_cover_in_warp_groups():
    from nbodyssey_b200.shard import shard_range
    for n in (1, 31, 32, 33, 1000, 20_001):
        for world in (1, 2, 3, 8):
            got = [shard_range(n, r, world) for r in range(world)]
            assert got[0][0] == 0 and got[-1][1] == n
            for (a0, a1, c), (b0, b1, _) in zip(got, got[1:]):
                assert a1 == b0
            for t0, t1, c in got:
                assert c % 32 == 0 and t1 - t0 <= c
                assert t0 % 32 == 0 or t0 == n
                assert t1 % 32 == 0 or t1 == n
