"""nb_compute_forces_naive_static: all-pairs forces for callers that cannot
allocate device memory (a host that owns every allocation, a fixed budget
reserved at start-up).  Its scratch is a fixed file-scope device array, so
this checks that the results equal those of the allocating entry point
(nb_compute_forces_dev, naive) within the all-pairs tolerance used by the
other GPU tests, over two calls in a row that reuse the same array, and that
sizes beyond the array's limit are refused before any GPU work.

Kept in a file collected last, so a stop-at-first-failure run has already
run every other test."""
import ctypes

import numpy as np
import pytest

from nbodyssey_b200 import _lib as L
from nbodyssey_b200 import api, ic

pytestmark = pytest.mark.gpu

MAX_N = 32768
EPS = 0.05


def rel_err(a, b):
    return np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)


def test_static_scratch_forces_match_allocating_path():
    torch = pytest.importorskip("torch")
    lib = L.load()
    assert api.device_count() >= 1
    ws = ctypes.c_void_p()
    L.check(lib.nb_workspace_create(ctypes.byref(ws)))
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    try:
        # two calls in a row on one device: the second reuses the array the
        # first left behind (different n, so stale contents would show)
        for n, seed in ((30_000, 31), (5_003, 32)):
            pos, _ = ic.two_disks(n, seed=seed)
            dpos = torch.from_numpy(pos).cuda()
            d_static = torch.full_like(dpos, float("nan"))
            d_ws = torch.zeros_like(dpos)
            L.check(lib.nb_compute_forces_naive_static(
                n, ctypes.c_void_p(dpos.data_ptr()),
                ctypes.c_void_p(d_static.data_ptr()), EPS, 1.0, stream))
            # the call's device status: no block gave up on its source tiles
            word = ctypes.c_uint(0xFFFFFFFF)
            L.check(lib.nb_compute_forces_naive_static_status(ctypes.byref(word), stream))
            assert word.value == 0
            prm = api.SimParams(epsilon=EPS, force="naive").to_c()
            L.check(lib.nb_compute_forces_dev(
                ws, n, ctypes.c_void_p(dpos.data_ptr()),
                ctypes.c_void_p(d_ws.data_ptr()), ctypes.byref(prm), stream))
            torch.cuda.synchronize()
            a = d_static.cpu().numpy().astype(np.float64)
            b = d_ws.cpu().numpy().astype(np.float64)
            assert np.all(np.isfinite(a)) and np.all(a[:, 3] == 0.0)
            r = rel_err(a[:, :3], b[:, :3])
            assert np.median(r) < 2e-6
            assert np.percentile(r, 99) < 2e-5
    finally:
        lib.nb_workspace_destroy(ws)


def test_static_scratch_rejects_sizes_beyond_its_limit():
    lib = L.load()
    dummy = ctypes.c_void_p(16)   # never dereferenced: the size check comes first
    rc = lib.nb_compute_forces_naive_static(MAX_N + 1, dummy, dummy, EPS, 1.0, None)
    assert rc == L.NB_ERR_INVALID
    assert b"32768" in lib.nb_last_error()
