"""Batched ensembles: many independent simulations advanced together.

All simulations' particles live in one set of device arrays and every phase of
a Barnes-Hut step is one kernel over all of them, so a step costs the same
dozen launches whether there are 2 simulations or 1,000 (captured once as a
CUDA graph).  Each simulation gets exactly the tree and interaction sets it
would get alone: its state after any number of steps is bit-identical to a
`Simulation` with the same parameters.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib as L
from .api import SimParams


class Ensemble:
    def __init__(self, states, params):
        """states: list of (pos4, vel4) float32 (n, 4) arrays; params: one
        SimParams for all, or a list with one per simulation (Barnes-Hut,
        all-pairs or AUTO, which picks by the tuned crossover)."""
        self._lib = L.load()
        if isinstance(params, SimParams):
            params = [params] * len(states)
        if len(params) != len(states):
            raise ValueError("one SimParams per simulation")
        self.n = [int(p.shape[0]) for p, _ in states]
        self.params = list(params)
        pos = np.ascontiguousarray(np.concatenate([p for p, _ in states]), np.float32)
        vel = np.ascontiguousarray(np.concatenate([v for _, v in states]), np.float32)
        ns = np.asarray(self.n, np.int32)
        cp = (L.nb_params * len(states))(*[p.to_c() for p in params])
        h = ctypes.c_void_p()
        L.check(self._lib.nb_ensemble_create(len(states), L.ptr(ns), L.ptr(pos),
                                             L.ptr(vel), cp, ctypes.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._lib.nb_ensemble_destroy(self._h)
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

    @property
    def nsims(self):
        return len(self.n)

    @property
    def particles(self):
        return int(sum(self.n))

    def step(self, nsteps=1):
        L.check(self._lib.nb_ensemble_step(self._h, int(nsteps)))

    def sync(self):
        L.check(self._lib.nb_ensemble_sync(self._h))

    def set_graphs(self, on=True):
        L.check(self._lib.nb_ensemble_set_graphs(self._h, 1 if on else 0))

    def state(self, sim):
        p = np.empty((self.n[sim], 4), np.float32)
        v = np.empty((self.n[sim], 4), np.float32)
        L.check(self._lib.nb_ensemble_get_state(self._h, int(sim), L.ptr(p), L.ptr(v)))
        return p, v

    def accelerations(self, sim):
        a = np.empty((self.n[sim], 4), np.float32)
        L.check(self._lib.nb_ensemble_get_accelerations(self._h, int(sim), L.ptr(a)))
        return a

    def energy(self):
        """(nsims, 3) array of (E, KE, PE)."""
        e = np.zeros((self.nsims, 3), np.float64)
        L.check(self._lib.nb_ensemble_energy(self._h, L.ptr(e)))
        return e

    def force(self, sim):
        """The force module simulation `sim` runs with, "naive" or "bh"
        (AUTO resolves by the tuned crossover inside a batch)."""
        f = ctypes.c_int()
        L.check(self._lib.nb_ensemble_force(self._h, int(sim), ctypes.byref(f)))
        return "naive" if f.value == L.NB_FORCE_NAIVE else "bh"

    def kernels_per_step(self):
        """Kernel launches of one step of this ensemble."""
        k = ctypes.c_int()
        L.check(self._lib.nb_ensemble_kernels_per_step(self._h, ctypes.byref(k)))
        return k.value

    def record(self, slot):
        L.check(self._lib.nb_ensemble_record(self._h, int(slot)))

    def elapsed_ms(self, a, b):
        ms = ctypes.c_double()
        L.check(self._lib.nb_ensemble_elapsed_ms(self._h, int(a), int(b), ctypes.byref(ms)))
        return ms.value


def shard(items, rank, world):
    """Deterministic split of independent simulations over `world` ranks
    (one process per GPU, no collective): greedy by particle count, largest
    first, so every rank gets a similar load.  Returns this rank's indices."""
    order = sorted(range(len(items)), key=lambda i: (-int(items[i]), i))
    load = [0] * world
    own = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        own[r].append(i)
        load[r] += int(items[i])
    return sorted(own[rank])
