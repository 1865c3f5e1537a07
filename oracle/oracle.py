"""CPU oracle for the nbodyssey force-and-step path (ctypes + NumPy).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
and by ``bench.py``'s CPU-baseline leg, never by the product package.

Two layers:

* ``libnboracle.so`` (oracle/nbody_oracle.c): the LBVH pipeline (Morton keys,
  stable sort, Karras build, centres of mass, thread and warp walks) in the
  device's exact float arithmetic, plus FP64 all-pairs force and energy with
  OpenMP.  Built by ``make -C oracle``.
* NumPy restatements of the reference's CPU integrator
  (scripts/reference_nbody.py:45-81): ``accelerations`` and ``total_energy``.

The oracle is pinned against fixtures produced by the reference's own Python
scripts (tests/golden/make_golden.py).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libnboracle.so")
_lib = None

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_i64 = ctypes.c_int64
_int = ctypes.c_int
_flt = ctypes.c_float
_vp = ctypes.c_void_p


def build():
    """Compile oracle/libnboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    L = ctypes.CDLL(_LIB_PATH)
    L.orc_num_threads.restype = _int
    L.orc_set_threads.argtypes = [_int]
    L.orc_bbox.argtypes = [_f32p, _i64, _f32p, _f32p]
    L.orc_morton.argtypes = [_f32p, _i64, _f32p, _f32p, _int, _u64p]
    L.orc_sort_pairs.argtypes = [_u64p, _i64, _int, _u64p, _u32p]
    L.orc_karras.argtypes = [_u64p, _i64, _int, _i32p, _i32p]
    L.orc_com.argtypes = [_f32p, _i64, _i32p, _f32p, _f32p, _f32p, _f32p, _f64p]
    _dbl = ctypes.c_double
    L.orc_walk_thread.argtypes = [_f32p, _i64, _i32p, _f32p, _f32p, _flt, _dbl,
                                  _flt, _i64p, _i64, _f64p, _i64p, _i32p]
    L.orc_walk_thread.restype = _int
    L.orc_walk_warp.argtypes = L.orc_walk_thread.argtypes
    L.orc_walk_warp.restype = _int
    L.orc_allpairs_f64.argtypes = [_f32p, _vp, _i64, _dbl, _flt, _vp, _i64, _f64p]
    L.orc_allpairs_f32.argtypes = [_f32p, _i64, _flt, _flt, _vp, _i64, _f32p]
    L.orc_energy_f64.argtypes = [_f32p, _vp, _f32p, _i64, _dbl, _flt, _f64p]
    L.orc_kick.argtypes = [_f32p, _f32p, _i64, _flt]
    L.orc_drift.argtypes = [_f32p, _f32p, _f32p, _i64, _flt, _int]
    _lib = L
    return L


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def num_threads():
    return lib().orc_num_threads()


def set_threads(t):
    lib().orc_set_threads(int(t))


# --------------------------------------------------------------------------
# LBVH pipeline
# --------------------------------------------------------------------------

def bbox(pos4):
    p = _c(pos4, np.float32)
    lo = np.zeros(3, np.float32)
    hi = np.zeros(3, np.float32)
    lib().orc_bbox(p, p.shape[0], lo, hi)
    return lo, hi


def morton_keys(pos4, key_bits=30, lo=None, hi=None):
    """Morton keys of float32 (x, y, z, m) rows (src/forces_bh.cu:202-220)."""
    p = _c(pos4, np.float32)
    if lo is None:
        lo, hi = bbox(p)
    keys = np.zeros(p.shape[0], np.uint64)
    lib().orc_morton(p, p.shape[0], _c(lo, np.float32), _c(hi, np.float32),
                     int(key_bits), keys)
    return keys


def sort_pairs(keys, key_bits=30):
    """Stable sort; returns (sorted keys, permutation of original indices)."""
    k = _c(keys, np.uint64)
    ko = np.zeros_like(k)
    perm = np.zeros(k.shape[0], np.uint32)
    lib().orc_sort_pairs(k, k.shape[0], int(key_bits), ko, perm)
    return ko, perm


def karras(keys_sorted, key_bits=30):
    """Returns children [n-1, 2] and parent [2n-1] (src/forces_bh.cu:242-277)."""
    k = _c(keys_sorted, np.uint64)
    n = k.shape[0]
    ch = np.zeros((max(n - 1, 0), 2), np.int32)
    par = np.zeros(max(2 * n - 1, 0), np.int32)
    lib().orc_karras(k, n, int(key_bits), ch, par)
    return ch, par


def centres_of_mass(pos_sorted4, children):
    """Returns com4 [n-1,4], size2 [n-1], box_lo [n-1,3], box_hi [n-1,3],
    fp64 sums [n-1,4] (src/forces_bh.cu:281-331)."""
    ps = _c(pos_sorted4, np.float32)
    n = ps.shape[0]
    ni = max(n - 1, 0)
    com = np.zeros((ni, 4), np.float32)
    size2 = np.zeros(ni, np.float32)
    lo = np.zeros((ni, 3), np.float32)
    hi = np.zeros((ni, 3), np.float32)
    sums = np.zeros((ni, 4), np.float64)
    lib().orc_com(ps, n, _c(children, np.int32), com, size2, lo, hi, sums)
    return com, size2, lo, hi, sums


class Tree:
    """A full LBVH built by the oracle for one set of float32 positions."""

    def __init__(self, pos4, key_bits=30):
        self.pos4 = _c(pos4, np.float32)
        self.n = self.pos4.shape[0]
        self.key_bits = key_bits
        self.lo, self.hi = bbox(self.pos4)
        self.keys = morton_keys(self.pos4, key_bits, self.lo, self.hi)
        self.keys_sorted, self.perm = sort_pairs(self.keys, key_bits)
        self.pos_sorted = np.ascontiguousarray(self.pos4[self.perm.astype(np.int64)])
        self.children, self.parent = karras(self.keys_sorted, key_bits)
        (self.com, self.size2, self.box_lo, self.box_hi,
         self.sums) = centres_of_mass(self.pos_sorted, self.children)

    def walk_thread(self, theta, eps, G=1.0, targets=None):
        """Per-thread walk for sorted targets.  Returns (acc [nt,3] fp64,
        interactions [nt], depth [nt])."""
        t = (np.arange(self.n, dtype=np.int64) if targets is None
             else _c(targets, np.int64))
        acc = np.zeros((t.shape[0], 3), np.float64)
        inter = np.zeros(t.shape[0], np.int64)
        depth = np.zeros(t.shape[0], np.int32)
        rc = lib().orc_walk_thread(self.pos_sorted, self.n, self.children,
                                   self.com, self.size2, float(theta),
                                   float(eps) ** 2, float(G), t, t.shape[0], acc,
                                   inter, depth)
        if rc != 0:
            raise RuntimeError("oracle walk stack overflow")
        return acc, inter, depth

    def walk_warp(self, theta, eps, G=1.0, warps=None):
        """Warp walk for the listed warps (32 sorted targets each).  Returns
        (acc [nw*32,3], interactions [nw], depth [nw])."""
        nwarps = (self.n + 31) // 32
        w = (np.arange(nwarps, dtype=np.int64) if warps is None
             else _c(warps, np.int64))
        acc = np.zeros((w.shape[0] * 32, 3), np.float64)
        inter = np.zeros(w.shape[0], np.int64)
        depth = np.zeros(w.shape[0], np.int32)
        rc = lib().orc_walk_warp(self.pos_sorted, self.n, self.children,
                                 self.com, self.size2, float(theta),
                                 float(eps) ** 2, float(G), w, w.shape[0], acc,
                                 inter, depth)
        if rc != 0:
            raise RuntimeError("oracle warp walk stack overflow")
        return acc, inter, depth

    def forces(self, theta, eps, G=1.0, traverse="thread"):
        """Accelerations in original particle order (fp64) plus per-particle
        interaction counts (warp mode: the warp's count for every lane)."""
        if traverse == "thread":
            acc_s, inter_s, _ = self.walk_thread(theta, eps, G)
        else:
            acc_w, inter_w, _ = self.walk_warp(theta, eps, G)
            acc_s = acc_w[: self.n]
            inter_s = np.repeat(inter_w, 32)[: self.n]
        acc = np.zeros((self.n, 3), np.float64)
        inter = np.zeros(self.n, np.int64)
        p = self.perm.astype(np.int64)
        acc[p] = acc_s
        inter[p] = inter_s
        return acc, inter


# --------------------------------------------------------------------------
# All-pairs, energy, integrator
# --------------------------------------------------------------------------

def allpairs_f64(pos4, eps, G=1.0, targets=None, pos_lo4=None):
    """Exact FP64 softened acceleration [nt, 3] (self term excluded); the
    softening enters as eps*eps in double."""
    p = _c(pos4, np.float32)
    n = p.shape[0]
    lo = None if pos_lo4 is None else _c(pos_lo4, np.float32)
    if targets is None:
        acc = np.zeros((n, 3), np.float64)
        lib().orc_allpairs_f64(p, None if lo is None else lo.ctypes.data, n,
                               float(eps) ** 2, float(G), None, n, acc)
        return acc
    t = _c(targets, np.int64)
    acc = np.zeros((t.shape[0], 3), np.float64)
    lib().orc_allpairs_f64(p, None if lo is None else lo.ctypes.data, n,
                           float(eps) ** 2, float(G), t.ctypes.data, t.shape[0],
                           acc)
    return acc


def allpairs_f32(pos4, eps, G=1.0, targets=None):
    """FP32 all-pairs with FP32 accumulation (the reference GPU precision)."""
    p = _c(pos4, np.float32)
    n = p.shape[0]
    if targets is None:
        acc = np.zeros((n, 4), np.float32)
        lib().orc_allpairs_f32(p, n, float(eps), float(G), None, n, acc)
        return acc
    t = _c(targets, np.int64)
    acc = np.zeros((t.shape[0], 4), np.float32)
    lib().orc_allpairs_f32(p, n, float(eps), float(G), t.ctypes.data,
                           t.shape[0], acc)
    return acc


def energy_f64(pos4, vel4, eps, G=1.0, pos_lo4=None):
    """Returns (E, KE, PE, Px, Py, Pz) in FP64."""
    p = _c(pos4, np.float32)
    v = _c(vel4, np.float32)
    out = np.zeros(6, np.float64)
    lo = None if pos_lo4 is None else _c(pos_lo4, np.float32)
    lib().orc_energy_f64(p, None if lo is None else lo.ctypes.data, v,
                         p.shape[0], float(eps) ** 2, float(G), out)
    return out


def kick(vel4, acc4, half_dt):
    v = _c(vel4, np.float32).copy()
    lib().orc_kick(v, _c(acc4, np.float32), v.shape[0], float(half_dt))
    return v


def drift(pos4, pos_lo4, vel4, dt, compensated=True):
    p = _c(pos4, np.float32).copy()
    lo = (np.zeros_like(p) if pos_lo4 is None else _c(pos_lo4, np.float32).copy())
    lib().orc_drift(p, lo, _c(vel4, np.float32), p.shape[0], float(dt),
                    1 if compensated else 0)
    return p, lo


# NumPy restatements of scripts/reference_nbody.py ---------------------------

def accelerations(pos, mass, eps2, G, chunk=2048, dtype=np.float64):
    """Softened acceleration on every particle, chunked over targets
    (scripts/reference_nbody.py:45-61): d = r_j - r_i, w = m_j / r^3 with
    r = sqrt(|d|^2 + eps2), a_i = G * sum_j w_ij d_ij."""
    pos = np.asarray(pos, dtype)
    mass = np.asarray(mass, dtype)
    n = pos.shape[0]
    out = np.empty((n, 3), dtype)
    one = dtype(1.0)
    for lo in range(0, n, chunk):
        hi = min(n, lo + chunk)
        d = pos[None, :, :] - pos[lo:hi, None, :]
        r = np.sqrt(np.sum(d * d, axis=2) + eps2)
        w = mass[None, :] * (one / (r * r * r))
        out[lo:hi] = np.einsum("bn,bnk->bk", w, d, dtype=dtype)
    return (G * out).astype(dtype)


def total_energy(pos, vel, mass, eps2, G, chunk=2048):
    """(E, KE, PE) in float64 (scripts/reference_nbody.py:64-81): KE from the
    velocities; PE as half the full double sum minus the self terms."""
    p = np.asarray(pos, np.float64)
    v = np.asarray(vel, np.float64)
    m = np.asarray(mass, np.float64)
    # numpy scalar types are kept as the reference keeps them (NEP 50: a
    # float32 eps2 / G stays float32 where the reference's does)
    ke = 0.5 * np.sum(m * np.sum(v * v, axis=1))
    total = 0.0
    n = p.shape[0]
    for lo in range(0, n, chunk):
        hi = min(n, lo + chunk)
        d = p[None, :, :] - p[lo:hi, None, :]
        inv = 1.0 / np.sqrt(np.sum(d * d, axis=2) + eps2)
        total += np.sum(m[lo:hi, None] * m[None, :] * inv)
    self_terms = np.sum(m * m) / np.sqrt(eps2)
    pe = -G * 0.5 * (total - self_terms)
    return ke + pe, ke, pe


def reference_loop(pos4, vel4, steps, dt, eps, G, dump_every, dtype,
                   chunk=2048):
    """The CPU integrator's run loop (scripts/reference_nbody.py:107-142),
    restated: a(x0), then per step kick / drift / a(x) / kick; a frame and an
    energy row after every step with step % dump_every == 0, and a final
    energy row labelled ``steps``.  Returns (frames, rows) with frames as
    float32 (n, 4) arrays and rows as (step, time, E, KE, PE, rel)."""
    eps2 = dtype(eps * eps)
    G_ = dtype(G)
    dt_ = dtype(dt)
    pos = np.asarray(pos4)[:, :3].astype(dtype)
    mass = np.asarray(pos4)[:, 3].astype(dtype)
    vel = np.asarray(vel4)[:, :3].astype(dtype)
    e0 = total_energy(pos, vel, mass, eps2, G_, chunk)[0]
    frames, rows = [], []

    def log(step):
        e, ke, pe = total_energy(pos, vel, mass, eps2, G_, chunk)
        rows.append((step, step * dt, e, ke, pe, (e - e0) / abs(e0)))

    acc = accelerations(pos, mass, eps2, G_, chunk, dtype)
    for step in range(steps):
        vel += dtype(0.5) * dt_ * acc
        pos += dt_ * vel
        acc = accelerations(pos, mass, eps2, G_, chunk, dtype)
        vel += dtype(0.5) * dt_ * acc
        if step % dump_every == 0:
            frames.append(np.column_stack([pos, mass]).astype("<f4"))
            log(step)
    log(steps)
    return frames, rows
