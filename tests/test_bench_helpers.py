"""bench.py's pure-Python helpers (CPU): the kernels-per-step count it claims
as gpu_launches and the committed ncu summaries it reads DRAM traffic from."""
import os

import bench


def test_kernels_per_step_matches_the_build_geometry():
    # prep, Morton keys, 4 sort passes, first build level, later levels, walk
    assert bench.bh_kernels_per_step(1000) == 1 + 1 + 4 + 1 + 0 + 1
    assert bench.bh_kernels_per_step(1_000_000) == 1 + 1 + 4 + 1 + 3 + 1   # 977 -> 66 -> 5 -> 1
    assert bench.bh_kernels_per_step(4_194_305) == 1 + 1 + 4 + 1 + 4 + 1
    assert bench.bh_kernels_per_step(1_000_000, key_bits=63) == 1 + 1 + 8 + 1 + 3 + 1


def test_profiled_traffic_follows_the_timed_semantics():
    warp = bench.profiled_traffic("k_walk_pair", "warp", 0.5)
    thread = bench.profiled_traffic("k_walk_pair", "thread", 0.5)
    assert warp is not None and thread is not None and thread != warp
    # only the captured workload (theta 0.5) has a capture
    assert bench.profiled_traffic("k_walk_pair", "warp", 0.3) is None
    assert bench.profiled_traffic("k_allpairs", "warp", 0.5) is None
    for name in ("walk_pair_1m.md", "walk_pair_thread_1m.md"):
        assert os.path.exists(os.path.join(bench.ROOT, "profiles", name))
