"""The autotuner on the GPU: the measured table is valid; NB_FORCE_AUTO takes
all-pairs below the tuned crossover and Barnes-Hut from it on, bit for bit
as the same method chosen by hand; a table set by hand gives the same bits
as the same table measured."""
import numpy as np
import pytest

from nbodyssey_b200 import _lib as L
from nbodyssey_b200 import api, ic

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tuned():
    base = api.tune_get()
    t = api.autotune()
    yield t
    api.tune_set(t if base["version"] else base)


def forces(pos, force, theta=0.5, traverse="warp"):
    prm = api.SimParams(epsilon=0.05, theta=theta, force=force, traverse=traverse)
    with api.Simulation(pos, np.zeros_like(pos), prm) as sim:
        return sim.compute_forces()


def test_measured_table_is_valid(tuned):
    assert tuned["version"] == L.NB_TUNE_VERSION and tuned["sms"] > 0
    for th, k in zip(tuned["ap_threads"], tuned["ap_k"]):
        assert th in (128, 256) and k in (2, 4, 8)
    assert tuned["walk_warps"] in (2, 4, 8)
    for row in tuned["crossover"]:
        for x in row:
            assert 2048 <= x <= 2 * 131072
    for x in tuned["crossover_batch"]:
        assert 1024 <= x <= 2 * 32768
    print("tuned table:", tuned)


@pytest.mark.parametrize("traverse", ["warp", "thread"])
def test_auto_follows_the_crossover(tuned, traverse):
    x = tuned["crossover"][1][1 if traverse == "warp" else 0]
    for n, method in ((max(x // 2, 64), "naive"), (x + 4096, "bh")):
        pos, _ = ic.two_disks(n, seed=71)
        a = forces(pos, "auto", traverse=traverse)
        b = forces(pos, method, traverse=traverse)
        assert np.array_equal(a, b), (n, method)


def test_table_by_hand_gives_the_same_bits(tuned):
    pos, _ = ic.two_disks(6000, seed=72)
    a = forces(pos, "naive")
    api.tune_set(dict(tuned))
    b = forces(pos, "naive")
    assert np.array_equal(a, b)
    # a different shape by hand: the same all-pairs sum to FP32 rounding
    other = dict(tuned)
    other["ap_threads"] = [128] * L.NB_TUNE_BUCKETS
    other["ap_k"] = [2] * L.NB_TUNE_BUCKETS
    other["ap_ctas"] = [4 * tuned["sms"]] * L.NB_TUNE_BUCKETS
    api.tune_set(other)
    try:
        c = forces(pos, "naive")
    finally:
        api.tune_set(dict(tuned))
    r = np.linalg.norm(c[:, :3] - a[:, :3], axis=1) / np.linalg.norm(a[:, :3], axis=1)
    assert r.max() < 1e-5
