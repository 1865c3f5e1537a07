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
