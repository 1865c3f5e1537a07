"""On-disk formats of the nbodyssey pipeline (docs/FORMATS.md:1-31).

All little-endian, float32:

* ``ic.bin``: int32 n, float4 pos[n] (x, y, z, m), float4 vel[n] (vx, vy, vz,
  0) -- read by src/main.cu:115-128, written by scripts/generate_ic.py:78-83.
* ``frame_%05d.bin``: int32 n, float4 pos[n] -- src/main.cu:130-138,
  scripts/reference_nbody.py:38-42.
* energy log CSV: header ``step,time,energy,kinetic,potential,rel_error`` and
  rows ``%d,%.5f,%.8e,%.8e,%.8e,%.3e`` (src/main.cu:160,176;
  scripts/reference_nbody.py:120,125).

The native run loop (``nb_run`` in the C ABI) writes the same files from C++;
these helpers serve the Python tools and the tests.
"""
from __future__ import annotations

import os
import struct

import numpy as np

ENERGY_HEADER = "step,time,energy,kinetic,potential,rel_error\n"


class FormatError(ValueError):
    """A file that is not a valid ic.bin / frame file (bad count, truncated)."""


def read_ic(path):
    """Returns (pos4, vel4) float32 arrays.  Raises FormatError on a
    non-positive count or a truncated file, as src/main.cu:118-126 does."""
    with open(path, "rb") as f:
        head = f.read(4)
        if len(head) < 4:
            raise FormatError("bad particle count in %s" % path)
        n = struct.unpack("<i", head)[0]
        if n <= 0:
            raise FormatError("bad particle count in %s" % path)
        body = f.read(32 * n)
    if len(body) < 32 * n:
        raise FormatError("truncated IC file: %s" % path)
    arr = np.frombuffer(body, "<f4")
    pos4 = arr[: 4 * n].reshape(n, 4).astype(np.float32)
    vel4 = arr[4 * n: 8 * n].reshape(n, 4).astype(np.float32)
    return pos4, vel4


def write_ic(path, pos4, vel4):
    pos4 = np.ascontiguousarray(pos4, "<f4")
    vel4 = np.ascontiguousarray(vel4, "<f4")
    if pos4.shape != vel4.shape or pos4.ndim != 2 or pos4.shape[1] != 4:
        raise FormatError("pos4 and vel4 must both be (n, 4)")
    with open(path, "wb") as f:
        f.write(struct.pack("<i", pos4.shape[0]))
        f.write(pos4.tobytes())
        f.write(vel4.tobytes())


def frame_bytes(pos4):
    pos4 = np.ascontiguousarray(pos4, "<f4")
    return struct.pack("<i", pos4.shape[0]) + pos4.tobytes()


def frame_name(index):
    return "frame_%05d.bin" % index


def write_frame(out_dir, index, pos4):
    path = os.path.join(out_dir, frame_name(index))
    with open(path, "wb") as f:
        f.write(frame_bytes(pos4))
    return path


def read_frame(path):
    with open(path, "rb") as f:
        data = f.read()
    if len(data) < 4:
        raise FormatError("bad frame file %s" % path)
    n = struct.unpack("<i", data[:4])[0]
    if n <= 0 or len(data) < 4 + 16 * n:
        raise FormatError("truncated frame file %s" % path)
    return np.frombuffer(data[4: 4 + 16 * n], "<f4").reshape(n, 4).copy()


def energy_row_py(step, time, e, ke, pe, rel):
    """One CSV row in the reference format."""
    return "%d,%.5f,%.8e,%.8e,%.8e,%.3e\n" % (step, time, e, ke, pe, rel)


def read_energy_csv(path):
    """Returns a structured array with the six columns."""
    return np.genfromtxt(path, delimiter=",", names=True)
