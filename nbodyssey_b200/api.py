"""Host-side mirror of the reference's force-and-step interface.

The reference (src/simulation.hpp, src/forces.cuh, src/integrator.cuh) is a
C++ API: ``SimParams`` / ``ForceMethod`` / ``BhTraversal``, a device-resident
``ParticleSystem``, ``compute_forces(sys, d_acc, p)``, ``leapfrog_step(sys,
d_acc, p)`` and ``total_energy(sys, p)``.  Here the same names sit on the C
ABI of libnbody_b200.so; all compute runs in the CUDA kernels of that library.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib as L


class ForceMethod:
    """src/simulation.hpp:4 (kNaive / kBarnesHut), plus AUTO: all-pairs below
    the measured crossover (NB_AUTO_CROSSOVER particles), Barnes-Hut above."""
    NAIVE = "naive"
    BARNES_HUT = "bh"
    AUTO = "auto"


class BhTraversal:
    """src/simulation.hpp:5 (kThread / kWarp)."""
    THREAD = "thread"
    WARP = "warp"


@dataclass
class SimParams:
    """src/simulation.hpp:8-15, with the reference CLI defaults
    (src/main.cu:25): dt 0.01, epsilon 0.05, G 1, theta 0.5, naive, thread.
    ``key_bits`` (30 or 63) and ``compensated`` (hi/lo positions through the
    drift) are this implementation's additions."""
    dt: float = 0.01
    epsilon: float = 0.05
    G: float = 1.0
    theta: float = 0.5
    force: str = ForceMethod.NAIVE
    traverse: str = BhTraversal.THREAD
    key_bits: int = 30
    compensated: bool = True
    walk_kernel: str = "pair"   # "pair" (child-pair records, default), "dfs" or "list"

    def to_c(self):
        if self.force not in (ForceMethod.NAIVE, ForceMethod.BARNES_HUT, ForceMethod.AUTO):
            raise ValueError("force must be naive, bh or auto, got: %r" % self.force)
        if self.traverse not in (BhTraversal.THREAD, BhTraversal.WARP):
            raise ValueError("traverse must be thread or warp, got: %r" % self.traverse)
        p = L.nb_params()
        p.dt = self.dt
        p.eps = self.epsilon
        p.G = self.G
        p.theta = self.theta
        p.force = {ForceMethod.NAIVE: L.NB_FORCE_NAIVE, ForceMethod.BARNES_HUT: L.NB_FORCE_BH,
                   ForceMethod.AUTO: L.NB_FORCE_AUTO}[self.force]
        p.traverse = L.NB_TRAVERSE_WARP if self.traverse == BhTraversal.WARP else L.NB_TRAVERSE_THREAD
        p.key_bits = int(self.key_bits)
        p.compensated = 1 if self.compensated else 0
        if self.walk_kernel not in ("pair", "dfs", "list"):
            raise ValueError("walk_kernel must be pair, dfs or list")
        p.walk_kernel = {"pair": 0, "dfs": 1, "list": 2}[self.walk_kernel]
        return p

    @classmethod
    def from_c(cls, p):
        """The SimParams of a C nb_params."""
        force = {L.NB_FORCE_NAIVE: ForceMethod.NAIVE, L.NB_FORCE_BH: ForceMethod.BARNES_HUT,
                 L.NB_FORCE_AUTO: ForceMethod.AUTO}[p.force]
        return cls(dt=p.dt, epsilon=p.eps, G=p.G, theta=p.theta, force=force,
                   traverse=BhTraversal.WARP if p.traverse == L.NB_TRAVERSE_WARP
                   else BhTraversal.THREAD,
                   key_bits=p.key_bits, compensated=bool(p.compensated),
                   walk_kernel={0: "pair", 1: "dfs", 2: "list"}[p.walk_kernel])


def _rows4(a, name):
    a = np.ascontiguousarray(a, dtype=np.float32)
    if a.ndim != 2 or a.shape[1] != 4:
        raise ValueError("%s must be an (n, 4) float32 array" % name)
    return a


def tune_table_dict(t):
    """A C nb_tune_table as a plain dict."""
    return {"version": t.version, "sms": t.sms, "device": t.device.decode(),
            "ap_threads": list(t.ap_threads), "ap_k": list(t.ap_k),
            "ap_ctas": list(t.ap_ctas), "walk_warps": t.walk_warps,
            "crossover": [list(r) for r in t.crossover],
            "crossover_batch": list(t.crossover_batch)}


def autotune(cache_path=None):
    """Measures the tuning table on the current device (all-pairs shape per
    size, walk warps per block, all-pairs / Barnes-Hut crossover per theta
    class and traversal), installs it and returns it as a dict."""
    t = L.nb_tune_table()
    L.check(L.load().nb_autotune(cache_path.encode() if cache_path else None,
                                 ctypes.byref(t)))
    return tune_table_dict(t)


def tune_get():
    t = L.nb_tune_table()
    L.check(L.load().nb_tune_get(ctypes.byref(t)))
    return tune_table_dict(t)


def tune_set(table: dict):
    """Installs a tuning table (a dict as tune_get returns) by hand."""
    t = L.nb_tune_table()
    L.check(L.load().nb_tune_defaults(ctypes.byref(t)))
    for k in ("ap_threads", "ap_k", "ap_ctas"):
        getattr(t, k)[:] = table[k]
    t.walk_warps = table["walk_warps"]
    for i in range(L.NB_TUNE_THETAS):
        t.crossover[i][:] = table["crossover"][i]
    if "crossover_batch" in table:
        t.crossover_batch[:] = table["crossover_batch"]
    L.check(L.load().nb_tune_set(ctypes.byref(t)))


def read_state(path):
    """A state file (checkpoint) or plain ic.bin: dict with pos, vel, lo, acc
    ((n, 4) float32), params (SimParams, None for a plain ic.bin) and flags
    (NB_STATE_* bits)."""
    lib = L.load()
    n = ctypes.c_int(0)
    L.check(lib.nb_read_state_file(path.encode(), ctypes.byref(n), None, None, None,
                                   None, None, None))
    pos, vel, lo, acc = (np.empty((n.value, 4), np.float32) for _ in range(4))
    prm = L.nb_params()
    flags = ctypes.c_int(0)
    L.check(lib.nb_read_state_file(path.encode(), ctypes.byref(n), L.ptr(pos), L.ptr(vel),
                                   L.ptr(lo), L.ptr(acc), ctypes.byref(prm),
                                   ctypes.byref(flags)))
    params = SimParams.from_c(prm) if flags.value & L.NB_STATE_TRAILER else None
    return {"pos": pos, "vel": vel, "lo": lo, "acc": acc, "params": params,
            "flags": flags.value}


def write_state(path, pos4, vel4, params: SimParams, lo4=None, acc4=None):
    """Writes a state file from host arrays (lo4 / acc4 may be None)."""
    pos4 = _rows4(pos4, "pos4")
    vel4 = _rows4(vel4, "vel4")
    lo4 = None if lo4 is None else _rows4(lo4, "lo4")
    acc4 = None if acc4 is None else _rows4(acc4, "acc4")
    L.check(L.load().nb_write_state_file(path.encode(), pos4.shape[0], L.ptr(pos4),
                                         L.ptr(vel4), L.ptr(lo4), L.ptr(acc4),
                                         ctypes.byref(params.to_c())))


def device_count():
    c = ctypes.c_int(0)
    L.check(L.load().nb_device_count(ctypes.byref(c)))
    return c.value


class Simulation:
    """One simulation whose state lives in HBM (ParticleSystem + integrator,
    src/simulation.cu:4-24, src/integrator.cu:27-37)."""

    def __init__(self, pos4, vel4, params: SimParams | None = None):
        self._lib = L.load()
        pos4 = _rows4(pos4, "pos4")
        vel4 = _rows4(vel4, "vel4")
        if pos4.shape != vel4.shape:
            raise ValueError("pos4 and vel4 must have the same shape")
        self.params = params or SimParams()
        self.n = pos4.shape[0]
        h = ctypes.c_void_p()
        L.check(self._lib.nb_sim_create(self.n, L.ptr(pos4), L.ptr(vel4),
                                        ctypes.byref(self.params.to_c()),
                                        ctypes.byref(h)))
        self._h = h

    # lifetime -------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            self._lib.nb_sim_destroy(self._h)
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

    # state ------------------------------------------------------------------
    def set_params(self, params: SimParams):
        L.check(self._lib.nb_set_params(self._h, ctypes.byref(params.to_c())))
        self.params = params

    def set_state(self, pos4, vel4):
        pos4 = _rows4(pos4, "pos4")
        vel4 = _rows4(vel4, "vel4")
        if pos4.shape[0] != self.n or vel4.shape[0] != self.n:
            raise ValueError("state must keep n = %d" % self.n)
        L.check(self._lib.nb_set_state(self._h, L.ptr(pos4), L.ptr(vel4)))

    @classmethod
    def from_state(cls, path):
        """A simulation resumed from a state file written by save_state: the
        stored parameters, positions with their low-order parts, velocities
        and a(x); it continues bit for bit as the run that wrote it."""
        st = read_state(path)
        sim = cls(st["pos"], st["vel"], st["params"] or SimParams())
        sim.load_state(path)
        return sim

    def save_state(self, path):
        """Checkpoint: the state file (ic.bin layout + trailer) of this
        simulation's current state."""
        L.check(self._lib.nb_save_state(self._h, path.encode()))

    def load_state(self, path):
        """Replaces the state (and, from a state file, the parameters)."""
        L.check(self._lib.nb_load_state(self._h, path.encode()))
        p = L.nb_params()
        L.check(self._lib.nb_get_params(self._h, ctypes.byref(p)))
        self.params = SimParams.from_c(p)

    def _get(self, fn):
        out = np.empty((self.n, 4), np.float32)
        L.check(fn(self._h, L.ptr(out)))
        return out

    def positions(self):
        """download_positions (src/simulation.cu:22-24)."""
        return self._get(self._lib.nb_get_positions)

    def velocities(self):
        return self._get(self._lib.nb_get_velocities)

    def accelerations(self):
        """The acceleration buffer: a(x) of the current positions after a
        step or compute_forces."""
        return self._get(self._lib.nb_get_accelerations)

    def set_state_acc(self, pos4, vel4, acc4):
        """Uploads a state with its a(x): the next step needs no priming
        force evaluation."""
        pos4 = _rows4(pos4, "pos4")
        vel4 = _rows4(vel4, "vel4")
        acc4 = _rows4(acc4, "acc4")
        if not (pos4.shape == vel4.shape == acc4.shape) or pos4.shape[0] != self.n:
            raise ValueError("pos4 / vel4 / acc4 must be (n, 4)")
        L.check(self._lib.nb_set_state_acc(self._h, L.ptr(pos4), L.ptr(vel4), L.ptr(acc4)))

    def position_lo(self):
        return self._get(self._lib.nb_get_position_lo)

    # compute ----------------------------------------------------------------
    def compute_forces(self):
        """compute_forces (src/forces.cu:68-86): a(x), original order."""
        return self._get(self._lib.nb_compute_forces)

    def step_host(self, pos4, vel4, acc4, out=None):
        """One leapfrog step of host-resident state: (pos, vel, a(x)) in,
        (pos, vel, a(x_new)) out (nb_step_host).  `out` may give the three
        output arrays (pinned ones avoid a staging copy)."""
        pos4 = _rows4(pos4, "pos4")
        vel4 = _rows4(vel4, "vel4")
        acc4 = _rows4(acc4, "acc4")
        if out is None:
            out = tuple(np.empty_like(pos4) for _ in range(3))
        L.check(self._lib.nb_step_host(self._h, L.ptr(pos4), L.ptr(vel4), L.ptr(acc4),
                                       L.ptr(out[0]), L.ptr(out[1]), L.ptr(out[2])))
        return out

    def step_host_state(self, pos4, vel4, out=None):
        """One leapfrog step of host-resident (pos, vel) (nb_step_host_state):
        a(x) and the low-order position parts stay on the device while the
        positions handed in are the ones the previous call returned."""
        pos4 = _rows4(pos4, "pos4")
        vel4 = _rows4(vel4, "vel4")
        if out is None:
            out = tuple(np.empty_like(pos4) for _ in range(2))
        L.check(self._lib.nb_step_host_state(self._h, L.ptr(pos4), L.ptr(vel4),
                                             L.ptr(out[0]), L.ptr(out[1])))
        return out

    def step(self, nsteps=1):
        """leapfrog_step x nsteps (asynchronous; see sync())."""
        L.check(self._lib.nb_step(self._h, int(nsteps)))

    def sync(self):
        L.check(self._lib.nb_sync(self._h))

    def energy(self):
        """total_energy (src/integrator.cu:93-110): (E, KE, PE)."""
        e = np.zeros(3, np.float64)
        L.check(self._lib.nb_energy(self._h, L.ptr(e), None))
        return float(e[0]), float(e[1]), float(e[2])

    def momentum(self):
        e = np.zeros(3, np.float64)
        m = np.zeros(3, np.float64)
        L.check(self._lib.nb_energy(self._h, L.ptr(e), L.ptr(m)))
        return m

    # timing -------------------------------------------------------------------
    def set_timing(self, on=True):
        L.check(self._lib.nb_set_timing(self._h, 1 if on else 0))

    def reset_timing(self):
        L.check(self._lib.nb_reset_timing(self._h))

    def force_timing(self):
        """(ms total, calls) (src/forces.cu:88-90)."""
        ms = ctypes.c_double()
        calls = ctypes.c_long()
        L.check(self._lib.nb_force_timing(self._h, ctypes.byref(ms), ctypes.byref(calls)))
        return ms.value, calls.value

    def phase_times(self):
        """{phase: ms accumulated}, steps timed (src/forces_bh.cu:529-539)."""
        ms = np.zeros(L.NB_PHASES, np.float64)
        calls = ctypes.c_long()
        L.check(self._lib.nb_phase_times(self._h, L.ptr(ms), ctypes.byref(calls)))
        return dict(zip(L.PHASE_NAMES, ms.tolist())), calls.value

    def record(self, slot):
        L.check(self._lib.nb_record(self._h, int(slot)))

    def elapsed_ms(self, a, b):
        ms = ctypes.c_double()
        L.check(self._lib.nb_elapsed_ms(self._h, int(a), int(b), ctypes.byref(ms)))
        return ms.value

    def set_graphs(self, on=True):
        L.check(self._lib.nb_set_graphs(self._h, 1 if on else 0))

    # debug / parity -----------------------------------------------------------
    def debug_lbvh(self):
        """Tree of the current positions: dict of keys (sorted), perm,
        children, parent, com4, size2."""
        n = self.n
        out = dict(keys=np.zeros(n, np.uint64), perm=np.zeros(n, np.uint32),
                   children=np.zeros((n - 1, 2), np.int32),
                   parent=np.zeros(2 * n - 1, np.int32),
                   com4=np.zeros((n - 1, 4), np.float32),
                   size2=np.zeros(n - 1, np.float32))
        L.check(self._lib.nb_debug_lbvh(
            self._h, L.ptr(out["keys"]), L.ptr(out["perm"]), L.ptr(out["children"]),
            L.ptr(out["parent"]), L.ptr(out["com4"]), L.ptr(out["size2"])))
        return out

    def debug_pairs(self):
        """The tree's child-pair records, (n - 1, 12) float32 (see
        nb_debug_pairs in include/nbody_b200.h)."""
        out = np.empty((self.n - 1, 12), np.float32)
        L.check(self._lib.nb_debug_pairs(self._h, L.ptr(out)))
        return out

    def debug_forces(self):
        """(acc4, interaction counts), original order."""
        acc = np.empty((self.n, 4), np.float32)
        cnt = np.zeros(self.n, np.int32)
        L.check(self._lib.nb_debug_forces(self._h, L.ptr(acc), L.ptr(cnt)))
        return acc, cnt

    def compare_forces(self):
        """compare_forces (src/main.cu:75-112): (max_rel, mean_rel) between
        the naive and Barnes-Hut modules on the current state."""
        mx = ctypes.c_double()
        mean = ctypes.c_double()
        L.check(self._lib.nb_compare_forces(self._h, ctypes.byref(mx), ctypes.byref(mean)))
        return mx.value, mean.value

    def run(self, steps, dump_every=5, out_dir=None, energy_log=None,
            timing=False):
        """The run loop of src/main.cu:140-215 (frames + energy CSV)."""
        st = L.nb_run_stats()
        L.check(self._lib.nb_run(
            self._h, int(steps), int(dump_every),
            out_dir.encode() if out_dir else None,
            energy_log.encode() if energy_log else None,
            1 if timing else 0, ctypes.byref(st)))
        return {"wall_s": st.wall_s, "force_ms": st.force_ms,
                "force_calls": st.force_calls, "frames": st.frames,
                "e0": st.e0, "e_final": st.e_final, "rel_final": st.rel_final,
                "phase_ms": dict(zip(L.PHASE_NAMES, list(st.phase_ms)))}


# Reference-named free functions ---------------------------------------------

def compute_forces(sim: Simulation):
    return sim.compute_forces()


def leapfrog_step(sim: Simulation):
    sim.step(1)


def total_energy(sim: Simulation):
    return sim.energy()
