"""One Barnes-Hut simulation split over several GPUs: one process per GPU,
``torch.distributed`` (NCCL) for the exchange.

The reference drives one GPU from one process (src/main.cu); this splits its
force evaluation (src/forces.cu:68-86 dispatching to src/forces_bh.cu:463-527)
across ranks.  Every rank holds the whole state and builds the whole tree
each step (the build is about a tenth of the step, and redundant building
needs no exchange before the walk); the walk, most of the step, is split by
Morton-sorted target: rank r walks the 32-aligned range

    [r C, min((r + 1) C, n)),   C = 32 ceil(ceil(n / 32) / R)

so every warp group of 32 targets (the unit of the warp walk's semantics)
stays on one rank.  One all-gather of the ranks' sorted-order accelerations
(16 bytes per particle) gives every rank the whole a(x), and the gather
kernel scatters it to original order with the closing kick.  Each rank's
state is bit-identical to the one-GPU run: same tree, same interaction sets,
same float operations, and the exchange only copies.

The orchestration (ranges, padding, exchange) is in ``ShardedSimulation``;
the device work is behind a small engine interface, ``NativeEngine`` on the
library (nb_forces_range_dev / nb_forces_gather_dev).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib as L
from .api import SimParams, _rows4


def shard_range(n, rank, world):
    """Sorted-target range [t0, t1) of `rank` and the padded chunk C."""
    warps = (n + 31) // 32
    chunk = 32 * ((warps + world - 1) // world)
    t0 = min(n, rank * chunk)
    t1 = min(n, (rank + 1) * chunk)
    return t0, t1, chunk


def _all_gather(out, inp, group):
    """out (world * C rows) <- every rank's inp (C rows), in rank order."""
    import torch.distributed as dist
    try:
        dist.all_gather_into_tensor(out, inp, group=group)
    except (RuntimeError, NotImplementedError, AttributeError):
        world = dist.get_world_size(group)
        dist.all_gather(list(out.chunk(world)), inp, group=group)


class NativeEngine:
    """Device state and kernels of one rank, on the current CUDA device."""

    def __init__(self, pos4, vel4, params: SimParams):
        import torch
        self.torch = torch
        self.lib = L.load()
        self.n = pos4.shape[0]
        self.p = params.to_c()
        dev = torch.device("cuda", torch.cuda.current_device())
        self.pos = torch.from_numpy(pos4).to(dev)
        self.vel = torch.from_numpy(vel4).to(dev)
        self.acc = torch.zeros_like(self.pos)
        self.lo = torch.zeros_like(self.pos) if params.compensated else None
        self.ws = ctypes.c_void_p()
        L.check(self.lib.nb_workspace_create(ctypes.byref(self.ws)))

    def alloc(self, rows):
        return self.torch.zeros((rows, 4), dtype=self.torch.float32, device=self.pos.device)

    def _stream(self):
        return ctypes.c_void_p(self.torch.cuda.current_stream().cuda_stream)

    @staticmethod
    def _ptr(t):
        return ctypes.c_void_p(t.data_ptr()) if t is not None else None

    def forces_range(self, t0, t1, part, kick):
        """part[:t1 - t0] = a of sorted targets [t0, t1); with `kick`, the
        opening kick and drift of every particle first."""
        L.check(self.lib.nb_forces_range_dev(
            self.ws, self.n, self._ptr(self.pos), self._ptr(self.lo),
            self._ptr(self.vel) if kick else None, self._ptr(self.acc),
            self._ptr(part), ctypes.byref(self.p), t0, t1, self._stream()))

    def gather(self, sorted_all, kick):
        """acc <- sorted_all[:n] in original order (+ closing kick)."""
        L.check(self.lib.nb_forces_gather_dev(
            self.ws, self.n, self._ptr(sorted_all), self._ptr(self.acc),
            self._ptr(self.vel) if kick else None, ctypes.byref(self.p),
            self._stream()))

    def state(self):
        self.torch.cuda.current_stream().synchronize()
        return (self.pos.cpu().numpy(), self.vel.cpu().numpy(), self.acc.cpu().numpy())

    def close(self):
        if self.ws:
            L.check(self.lib.nb_workspace_destroy(self.ws))
            self.ws = ctypes.c_void_p()


class ShardedSimulation:
    """A simulation whose Barnes-Hut walk is split over the ranks of
    `group` (the default process group; one rank without one).  Same
    stepping as ``api.Simulation``: a(x) before the first step, then
    kick-drift-kick."""

    def __init__(self, pos4, vel4, params: SimParams, group=None, engine=None):
        pos4 = _rows4(pos4, "pos4")
        vel4 = _rows4(vel4, "vel4")
        if pos4.shape != vel4.shape:
            raise ValueError("pos4 and vel4 must have the same shape")
        self.group = group
        self.rank, self.world = 0, 1
        try:
            import torch.distributed as dist
            if dist.is_available() and dist.is_initialized():
                self.rank = dist.get_rank(group)
                self.world = dist.get_world_size(group)
        except ImportError:
            pass
        self.n = pos4.shape[0]
        self.t0, self.t1, self.chunk = shard_range(self.n, self.rank, self.world)
        self.engine = engine if engine is not None else NativeEngine(pos4, vel4, params)
        self.part = self.engine.alloc(self.chunk)
        self.sorted = self.engine.alloc(self.chunk * self.world)
        self.primed = False

    def _exchange(self):
        if self.world > 1:
            _all_gather(self.sorted, self.part, self.group)
        else:
            self.sorted[: self.chunk] = self.part

    def compute_forces(self):
        """a(x) of the current state on every rank."""
        self.engine.forces_range(self.t0, self.t1, self.part, kick=False)
        self._exchange()
        self.engine.gather(self.sorted, kick=False)
        self.primed = True

    def step(self, nsteps=1):
        if not self.primed:
            self.compute_forces()
        for _ in range(int(nsteps)):
            self.engine.forces_range(self.t0, self.t1, self.part, kick=True)
            self._exchange()
            self.engine.gather(self.sorted, kick=True)

    def state(self):
        """(positions, velocities, accelerations) as numpy arrays."""
        return self.engine.state()

    def close(self):
        close = getattr(self.engine, "close", None)
        if close:
            close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
