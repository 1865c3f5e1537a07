"""Simulation request server with continuous batching (nb_server_* C ABI).

    srv = Server(hbm_budget_bytes=8 << 30)
    rid = srv.submit(pos4, vel4, SimParams(force="bh", ...), steps=500,
                     dump_every=50, out_dir=None)
    srv.wait(rid); pos, vel = srv.result(rid)

Requests are admitted whenever their footprint fits the free part of the
device slot pool; all running simulations advance together, one set of
launches per step.  Each result is bit-identical to running the request alone
through `Simulation`.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib as L
from .api import SimParams

QUEUED, RUNNING, DONE, FAILED = 0, 1, 2, 3


class nb_server_stats(ctypes.Structure):
    _fields_ = [("completed", ctypes.c_longlong), ("failed", ctypes.c_longlong),
                ("queued", ctypes.c_longlong), ("running", ctypes.c_longlong),
                ("engine_steps", ctypes.c_longlong), ("particle_steps", ctypes.c_double),
                ("frames", ctypes.c_longlong), ("frame_bytes", ctypes.c_longlong),
                ("busy_s", ctypes.c_double), ("peak_running", ctypes.c_int),
                ("capacity_slots", ctypes.c_longlong), ("used_slots", ctypes.c_longlong)]


class Server:
    def __init__(self, hbm_budget_bytes=4 << 30, max_sims=1023):
        self._lib = L.load()
        h = ctypes.c_void_p()
        L.check(self._lib.nb_server_create(int(hbm_budget_bytes), int(max_sims),
                                           ctypes.byref(h)))
        self._h = h
        self._n = {}

    def close(self):
        if getattr(self, "_h", None):
            self._lib.nb_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, pos4, vel4, params: SimParams, steps, dump_every=0,
               out_dir=None):
        pos4 = np.ascontiguousarray(pos4, np.float32)
        vel4 = np.ascontiguousarray(vel4, np.float32)
        rid = ctypes.c_longlong()
        L.check(self._lib.nb_server_submit(
            self._h, pos4.shape[0], L.ptr(pos4), L.ptr(vel4),
            ctypes.byref(params.to_c()), int(steps), int(dump_every),
            out_dir.encode() if out_dir else None, ctypes.byref(rid)))
        self._n[rid.value] = pos4.shape[0]
        return rid.value

    def poll(self, rid):
        """(state, t_submit, t_admit, t_done), times in seconds since start."""
        st = ctypes.c_int()
        a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        L.check(self._lib.nb_server_poll(self._h, int(rid), ctypes.byref(st),
                                         ctypes.byref(a), ctypes.byref(b),
                                         ctypes.byref(c)))
        return st.value, a.value, b.value, c.value

    def wait(self, rid, timeout_s=600.0):
        L.check(self._lib.nb_server_wait(self._h, int(rid), float(timeout_s)))

    def force(self, rid):
        """The force module request `rid` runs with, "naive" or "bh"."""
        f = ctypes.c_int()
        L.check(self._lib.nb_server_force(self._h, int(rid), ctypes.byref(f)))
        return "naive" if f.value == L.NB_FORCE_NAIVE else "bh"

    def result(self, rid, release=True):
        if rid not in self._n:   # let the library report the unknown id
            L.check(self._lib.nb_server_result(self._h, int(rid), None, None, 0))
        n = self._n[rid]
        p = np.empty((n, 4), np.float32)
        v = np.empty((n, 4), np.float32)
        L.check(self._lib.nb_server_result(self._h, int(rid), L.ptr(p), L.ptr(v),
                                           1 if release else 0))
        if release:
            del self._n[rid]
        return p, v

    def stats(self):
        s = nb_server_stats()
        L.check(self._lib.nb_server_get_stats(self._h, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in nb_server_stats._fields_}
