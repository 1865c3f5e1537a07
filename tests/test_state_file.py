"""State files (checkpoint / resume), host side: the file starts with the
ic.bin layout of docs/FORMATS.md:8-16, so an ic.bin reader (the reference's
load_ic, src/main.cu:115-128, and formats.read_ic here) takes it as initial
conditions; the trailer carries the run's parameters, the low-order position
parts and a(x).  No GPU: these are the host-only entry points."""
import numpy as np
import pytest

from nbodyssey_b200 import _lib as L
from nbodyssey_b200 import api, formats


def _arrays(n, seed):
    rng = np.random.default_rng(seed)
    return [rng.standard_normal((n, 4)).astype(np.float32) for _ in range(4)]


def test_state_file_round_trip(tmp_path):
    pos, vel, lo, acc = _arrays(1001, 1)
    prm = api.SimParams(dt=0.005, epsilon=0.01, theta=0.3, force="bh", traverse="warp",
                        key_bits=63, compensated=True, walk_kernel="pair")
    path = str(tmp_path / "state.bin")
    api.write_state(path, pos, vel, prm, lo4=lo, acc4=acc)
    st = api.read_state(path)
    for k, a in (("pos", pos), ("vel", vel), ("lo", lo), ("acc", acc)):
        assert np.array_equal(st[k], a), k
    assert st["flags"] == L.NB_STATE_TRAILER | L.NB_STATE_ACC | L.NB_STATE_LO
    assert bytes(st["params"].to_c()) == bytes(prm.to_c())   # float32 fields
    # the ic.bin prefix: byte for byte what write_ic writes
    formats.write_ic(str(tmp_path / "ic.bin"), pos, vel)
    head = open(str(tmp_path / "ic.bin"), "rb").read()
    assert open(path, "rb").read()[: len(head)] == head
    p2, v2 = formats.read_ic(path)
    assert np.array_equal(p2, pos) and np.array_equal(v2, vel)


def test_state_file_without_acc(tmp_path):
    pos, vel, _, _ = _arrays(64, 2)
    path = str(tmp_path / "s.bin")
    api.write_state(path, pos, vel, api.SimParams())
    st = api.read_state(path)
    assert st["flags"] == L.NB_STATE_TRAILER
    assert not st["lo"].any() and not st["acc"].any()


def test_plain_ic_reads_as_state(tmp_path):
    pos, vel, _, _ = _arrays(77, 3)
    path = str(tmp_path / "ic.bin")
    formats.write_ic(path, pos, vel)
    st = api.read_state(path)
    assert st["flags"] == 0 and st["params"] is None
    assert np.array_equal(st["pos"], pos) and np.array_equal(st["vel"], vel)
    assert not st["lo"].any() and not st["acc"].any()


def test_truncated_trailer_is_an_io_error(tmp_path):
    pos, vel, lo, acc = _arrays(100, 4)
    path = str(tmp_path / "s.bin")
    api.write_state(path, pos, vel, api.SimParams(), lo4=lo, acc4=acc)
    data = open(path, "rb").read()
    open(path, "wb").write(data[:-17])
    with pytest.raises(L.NbError) as ei:
        api.read_state(path)
    assert ei.value.code == L.NB_ERR_IO
