"""Tuning table, host side: defaults, validation of tables set by hand, cache
files (save / load round trip; a missing or foreign file is NOT FOUND).  No
GPU: nothing here measures."""
import ctypes

import pytest

from nbodyssey_b200 import _lib as L
from nbodyssey_b200 import api


def test_defaults_are_the_fixed_b200_shapes():
    t = L.nb_tune_table()
    L.check(L.load().nb_tune_defaults(ctypes.byref(t)))
    assert t.version == L.NB_TUNE_VERSION
    assert set(t.ap_threads) == {256} and set(t.ap_k) == {4}
    assert t.walk_warps == 4
    assert all(x == L.NB_AUTO_CROSSOVER for r in t.crossover for x in r)


def test_invalid_tables_are_rejected():
    lib = L.load()
    t = L.nb_tune_table()
    L.check(lib.nb_tune_defaults(ctypes.byref(t)))
    t.ap_k[3] = 3   # not a compiled shape
    assert lib.nb_tune_set(ctypes.byref(t)) == L.NB_ERR_INVALID
    L.check(lib.nb_tune_defaults(ctypes.byref(t)))
    t.walk_warps = 5
    assert lib.nb_tune_set(ctypes.byref(t)) == L.NB_ERR_INVALID
    L.check(lib.nb_tune_defaults(ctypes.byref(t)))
    t.version = 99
    assert lib.nb_tune_set(ctypes.byref(t)) == L.NB_ERR_INVALID


def test_set_get_save_load_round_trip(tmp_path):
    base = api.tune_get()
    try:
        table = dict(base)
        table["ap_threads"] = [128] * L.NB_TUNE_BUCKETS
        table["ap_k"] = [8] * L.NB_TUNE_BUCKETS
        table["crossover"] = [[11000, 17000], [13000, 19000], [15000, 21000]]
        api.tune_set(table)
        got = api.tune_get()
        assert got["ap_threads"] == table["ap_threads"] and got["crossover"] == table["crossover"]
        path = str(tmp_path / "tune.bin")
        L.check(L.load().nb_tune_save(path.encode()))
        api.tune_set(base)
        L.check(L.load().nb_tune_load(path.encode()))
        assert api.tune_get()["crossover"] == table["crossover"]
    finally:
        api.tune_set(base)


def test_missing_cache_is_not_found(tmp_path):
    rc = L.load().nb_tune_load(str(tmp_path / "none.bin").encode())
    assert rc == L.NB_ERR_NOTFOUND


def test_foreign_cache_is_not_found(tmp_path):
    t = L.nb_tune_table()
    L.check(L.load().nb_tune_defaults(ctypes.byref(t)))
    t.device = b"some other GPU"
    path = tmp_path / "foreign.bin"
    path.write_bytes(bytes(t))
    assert L.load().nb_tune_load(str(path).encode()) == L.NB_ERR_NOTFOUND
