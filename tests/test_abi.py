"""The C-ABI library loads and exports every symbol include/nbody_b200.h
declares; host-only entry points (formats, argument checks) work without a
GPU.  No compute calls here."""
import ctypes
import os
import re

import numpy as np
import pytest

from nbodyssey_b200 import _lib as L
from nbodyssey_b200 import formats

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            names |= set(re.findall(r"^NB_API\s+[\w\s\*]*?\b(nb_\w+)\s*\(", text,
                                    flags=re.M))
    return sorted(names)


def test_header_declares_symbols():
    assert len(header_symbols()) >= 30


def test_every_declared_symbol_is_exported():
    lib = L.load()
    missing = [s for s in header_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_bindings_cover_header():
    assert set(header_symbols()) <= set(L.SIGNATURES)


def test_params_default_matches_reference_defaults():
    p = L.nb_params()
    L.load().nb_params_default(ctypes.byref(p))
    # src/main.cu:25, src/simulation.hpp:11-14
    assert abs(p.dt - 0.01) < 1e-9 and abs(p.eps - 0.05) < 1e-9
    assert p.G == 1.0 and abs(p.theta - 0.5) < 1e-9
    assert p.force == L.NB_FORCE_NAIVE and p.traverse == L.NB_TRAVERSE_THREAD


def _create(n, eps=0.05, theta=0.5, key_bits=30, force=0):
    lib = L.load()
    p = L.nb_params()
    lib.nb_params_default(ctypes.byref(p))
    p.eps, p.theta, p.key_bits, p.force = eps, theta, key_bits, force
    pos = np.zeros((max(n, 1), 4), np.float32)
    h = ctypes.c_void_p()
    rc = lib.nb_sim_create(n, L.ptr(pos), L.ptr(pos), ctypes.byref(p), ctypes.byref(h))
    return rc


@pytest.mark.parametrize("kw", [dict(n=0), dict(n=-3), dict(n=8, eps=0.0),
                                dict(n=8, eps=-1.0), dict(n=8, theta=-0.1),
                                dict(n=8, key_bits=32), dict(n=8, force=5)])
def test_invalid_arguments_rejected_before_any_device_work(kw):
    rc = _create(**kw)
    assert rc == L.NB_ERR_INVALID
    assert L.load().nb_last_error()


def test_energy_row_format_matches_main_cu():
    buf = ctypes.create_string_buffer(256)
    lib = L.load()
    assert lib.nb_format_energy_row(buf, 256, 10, 0.01, -0.1178, 0.58, -0.7, -0.1179) == 0
    row = buf.value.decode()
    # "%d,%.5f,%.8e,%.8e,%.8e,%.3e\n" (src/main.cu:176)
    t = np.float32(10) * np.float32(0.01)
    assert row == "%d,%.5f,%.8e,%.8e,%.8e,%.3e\n" % (
        10, float(t), -0.1178, 0.58, -0.7, (-0.1178 + 0.1179) / 0.1179)


def test_energy_row_matches_reference_csv(golden_dir):
    """Rows of reference_nbody.py's float64 CSV reformatted by the C ABI."""
    g = np.load(os.path.join(golden_dir, "refnbody.npz"))
    text = g["csv_float64"].tobytes().decode().splitlines()
    assert text[0] + "\n" == formats.ENERGY_HEADER
    e0 = None
    lib = L.load()
    for line in text[1:]:
        step, t, e, ke, pe, rel = line.split(",")
        e, ke, pe = float(e), float(ke), float(pe)
        if e0 is None:
            # recover E0 from the first row's printed rel error
            e0 = e / (1.0 + float(rel)) if float(rel) != 0 else e
        buf = ctypes.create_string_buffer(256)
        assert lib.nb_format_energy_row(buf, 256, int(step), 0.01, e, ke, pe, e0) == 0
        got = buf.value.decode().rstrip("\n").split(",")
        assert got[:5] == line.split(",")[:5]


def test_ic_roundtrip_and_errors(tmp_path, golden_dir):
    g = np.load(os.path.join(golden_dir, "refnbody.npz"))
    p = tmp_path / "ic.bin"
    p.write_bytes(g["ic_bytes"].tobytes())
    lib = L.load()
    n = ctypes.c_int(0)
    assert lib.nb_read_ic(str(p).encode(), ctypes.byref(n), None, None) == 0
    assert n.value == 512
    pos = np.zeros((512, 4), np.float32)
    vel = np.zeros((512, 4), np.float32)
    assert lib.nb_read_ic(str(p).encode(), ctypes.byref(n), L.ptr(pos), L.ptr(vel)) == 0
    assert np.array_equal(pos, g["pos4"]) and np.array_equal(vel, g["vel4"])
    # python reader agrees
    pp, vv = formats.read_ic(str(p))
    assert np.array_equal(pp, pos) and np.array_equal(vv, vel)
    # write back byte-identical
    q = tmp_path / "ic2.bin"
    assert lib.nb_write_ic(str(q).encode(), 512, L.ptr(pos), L.ptr(vel)) == 0
    assert q.read_bytes() == p.read_bytes()
    # truncated and bad-count files are errors (src/main.cu:118-126)
    t = tmp_path / "trunc.bin"
    t.write_bytes(p.read_bytes()[:1000])
    assert lib.nb_read_ic(str(t).encode(), ctypes.byref(n), L.ptr(pos), L.ptr(vel)) == L.NB_ERR_IO
    b = tmp_path / "bad.bin"
    b.write_bytes(np.int32(-4).tobytes())
    assert lib.nb_read_ic(str(b).encode(), ctypes.byref(n), None, None) == L.NB_ERR_IO
    assert lib.nb_read_ic(b"/nonexistent/x.bin", ctypes.byref(n), None, None) == L.NB_ERR_IO
    with pytest.raises(formats.FormatError):
        formats.read_ic(str(t))


def test_frame_bytes_match_reference(tmp_path, golden_dir):
    g = np.load(os.path.join(golden_dir, "refnbody.npz"))
    fr = g["frames_float64"][1]
    pos = np.frombuffer(fr.tobytes()[4:], np.float32).reshape(-1, 4).copy()
    lib = L.load()
    assert lib.nb_write_frame(str(tmp_path).encode(), 1, pos.shape[0], L.ptr(pos)) == 0
    assert (tmp_path / "frame_00001.bin").read_bytes() == fr.tobytes()
    assert formats.frame_bytes(pos) == fr.tobytes()
    assert g["frame_names_float64"][1] == formats.frame_name(1)


def test_device_count_without_gpu_is_not_an_error():
    c = ctypes.c_int(-1)
    assert L.load().nb_device_count(ctypes.byref(c)) == 0
    assert c.value >= 0
