"""Seeded initial conditions: two exponential disks on a collision course.

Follows the structure of the reference generator (scripts/generate_ic.py:
16-83: Gamma(2, R_d) radii with the tail resampled, a Gaussian vertical
profile, circular speeds from the enclosed mass under the softened monopole
force, a tilt about x, bulk velocities) with the recipe the benchmarks use:

* R_d = 1 truncated at R = 5; sigma_z = 0.1;
* enclosed mass from the analytic truncated exponential disk,
  M(<R) = M [1 - (1 + R/R_d) e^{-R/R_d}] / [1 - (1 + 5) e^{-5}];
* v_c(R) = sqrt(G M(<R) R^2 / (R^2 + eps^2)^{3/2}), plus an isotropic
  Gaussian dispersion of 0.05 v_c per component;
* disk A at (-10, -b/2, 0) moving +v along x, spin +1; disk B at
  (+10, +b/2, 0) moving -v, spin -1, tilted about x;
* optional Plummer core per galaxy (a fraction of its mass, scale a) with
  isotropic velocities drawn from the Plummer distribution function by the
  rejection method of Aarseth, Henon & Wielen (1974).

Equal particle masses: a galaxy of mass M with k particles has m = M / k.
Output rows are float32 (x, y, z, m) / (vx, vy, vz, 0), galaxy A first, the
``ic.bin`` layout of docs/FORMATS.md.
"""
from __future__ import annotations

import math

import numpy as np


def _exp_disk_menc(r, rd, rmax, mass):
    norm = 1.0 - (1.0 + rmax / rd) * math.exp(-rmax / rd)
    x = r / rd
    return mass * (1.0 - (1.0 + x) * np.exp(-x)) / norm


def _plummer_menc(r, a, mass):
    return mass * r ** 3 / (r * r + a * a) ** 1.5


def _plummer(n, mass, a, G, rng):
    """Positions and velocities of an isotropic Plummer sphere."""
    x1 = rng.uniform(0.0, 0.99, size=n)   # mass fraction, far tail cut
    r = a / np.sqrt(x1 ** (-2.0 / 3.0) - 1.0)
    u = rng.normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=1)[:, None]
    pos = u * r[:, None]
    # speed fraction q of the local escape speed: g(q) = q^2 (1 - q^2)^3.5
    q = np.empty(n)
    todo = np.arange(n)
    while todo.size:
        qq = rng.uniform(0.0, 1.0, size=todo.size)
        yy = rng.uniform(0.0, 0.1, size=todo.size)
        ok = yy < qq * qq * (1.0 - qq * qq) ** 3.5
        q[todo[ok]] = qq[ok]
        todo = todo[~ok]
    vesc = np.sqrt(2.0 * G * mass / np.sqrt(r * r + a * a))
    w = rng.normal(size=(n, 3))
    w /= np.linalg.norm(w, axis=1)[:, None]
    vel = w * (q * vesc)[:, None]
    return pos, vel


def galaxy(n, mass, center, bulk, inclination_deg, spin, eps, rng, G=1.0,
           rd=1.0, rmax=5.0, sigma_z=0.1, dispersion=0.05, core_frac=0.0,
           core_a=0.1):
    """One galaxy of n particles: an exponential disk plus an optional
    Plummer core holding ``core_frac`` of the mass."""
    n_core = int(round(n * core_frac)) if core_frac > 0 else 0
    n_disk = n - n_core
    m = mass / n
    m_core = m * n_core
    m_disk = m * n_disk

    r = rng.gamma(2.0, rd, size=n_disk)
    over = r > rmax
    while np.any(over):
        r[over] = rng.gamma(2.0, rd, size=int(over.sum()))
        over = r > rmax
    phi = rng.uniform(0.0, 2.0 * np.pi, size=n_disk)
    z = rng.normal(0.0, sigma_z, size=n_disk)
    menc = _exp_disk_menc(r, rd, rmax, m_disk)
    if n_core:
        menc = menc + _plummer_menc(r, core_a, m_core)
    vc = np.sqrt(G * menc * r * r / (r * r + eps * eps) ** 1.5)
    pos = np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=1)
    vel = np.stack([-spin * vc * np.sin(phi), spin * vc * np.cos(phi),
                    np.zeros(n_disk)], axis=1)
    vel += rng.normal(size=(n_disk, 3)) * (dispersion * vc)[:, None]
    if n_core:
        cp, cv = _plummer(n_core, m_core, core_a, G, rng)
        pos = np.concatenate([cp, pos])
        vel = np.concatenate([cv, vel])
    if inclination_deg:
        c = math.cos(math.radians(inclination_deg))
        s = math.sin(math.radians(inclination_deg))
        rot = np.array([[1.0, 0.0, 0.0], [0.0, c, -s], [0.0, s, c]])
        pos = pos @ rot.T
        vel = vel @ rot.T
    pos += np.asarray(center, np.float64)
    vel += np.asarray(bulk, np.float64)
    pos4 = np.column_stack([pos, np.full(n, m)]).astype(np.float32)
    vel4 = np.column_stack([vel, np.zeros(n)]).astype(np.float32)
    return pos4, vel4


def two_disks(n_total, seed=0, eps=0.05, mass_ratio=1.0, impact=4.0,
              separation=20.0, approach=0.25, inclination_deg=30.0,
              core_frac=0.0, core_a=0.1, G=1.0):
    """Two galaxies, A (mass 1) and B (mass ``mass_ratio``), equal particle
    masses, n_total particles split in proportion to mass."""
    rng = np.random.default_rng(seed)
    n_a = int(round(n_total / (1.0 + mass_ratio)))
    n_b = n_total - n_a
    pa, va = galaxy(n_a, 1.0, [-separation / 2, -impact / 2, 0.0],
                    [approach, 0.0, 0.0], 0.0, +1.0, eps, rng, G=G,
                    core_frac=core_frac, core_a=core_a)
    pb, vb = galaxy(n_b, mass_ratio, [separation / 2, impact / 2, 0.0],
                    [-approach, 0.0, 0.0], inclination_deg, -1.0, eps, rng,
                    G=G, core_frac=core_frac, core_a=core_a)
    return np.concatenate([pa, pb]), np.concatenate([va, vb])


def plain_config(n_total=12000, seed=0):
    """The plain all-pairs workload: N=12,000, eps 0.05, dt 0.005."""
    return two_disks(n_total, seed=seed)


def bh_config(n_total=1_000_000, seed=0):
    """The Barnes-Hut workload: N=1,000,000, same recipe."""
    return two_disks(n_total, seed=seed)


def precision_config(n_total=262_144, seed=0):
    """The precision study: a 10 % Plummer core (a = 0.1) per galaxy, used
    with eps 0.01, dt 0.002."""
    return two_disks(n_total, seed=seed, eps=0.01, core_frac=0.1, core_a=0.1)


def ensemble_specs(count, seed=0, n_lo=2048, n_hi=131072):
    """Encounter parameters of a batched ensemble: N log-uniform in
    [n_lo, n_hi] rounded to a multiple of 32, mass ratio U[0.25, 1], impact
    parameter U[2, 8], disk-B inclination U[0, 90] degrees, approach speed
    U[0.3, 0.7]."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        n = math.exp(rng.uniform(math.log(n_lo), math.log(n_hi)))
        n = max(32, int(round(n / 32.0)) * 32)
        out.append(dict(n=n, mass_ratio=float(rng.uniform(0.25, 1.0)),
                        impact=float(rng.uniform(2.0, 8.0)),
                        inclination_deg=float(rng.uniform(0.0, 90.0)),
                        approach=float(rng.uniform(0.3, 0.7)),
                        seed=int(rng.integers(0, 2 ** 31 - 1))))
    return out


def from_spec(spec, eps=0.05):
    return two_disks(spec["n"], seed=spec["seed"], eps=eps,
                     mass_ratio=spec["mass_ratio"], impact=spec["impact"],
                     approach=spec["approach"],
                     inclination_deg=spec["inclination_deg"])


def main(argv=None):
    """Write a two-disk ``ic.bin``.  The flags carry the reference
    generator's names (scripts/generate_ic.py:89-103); the defaults are this
    module's benchmark recipe, and ``--mass-ratio`` / ``--core-frac`` /
    ``--core-a`` reach the mass-ratio and Plummer-core variants."""
    import argparse

    from . import formats

    ap = argparse.ArgumentParser(description="Two exponential disks on a "
                                 "collision course -> ic.bin")
    ap.add_argument("--particles", type=int, default=40000)
    ap.add_argument("--out", default="ic.bin")
    ap.add_argument("--separation", type=float, default=20.0)
    ap.add_argument("--impact", type=float, default=4.0)
    ap.add_argument("--approach", type=float, default=0.25)
    ap.add_argument("--mass-ratio", type=float, default=1.0)
    ap.add_argument("--eps", type=float, default=0.05)
    ap.add_argument("--inclination", type=float, default=30.0)
    ap.add_argument("--core-frac", type=float, default=0.0)
    ap.add_argument("--core-a", type=float, default=0.1)
    ap.add_argument("--seed", type=int, default=0)
    a = ap.parse_args(argv)
    if a.particles < 2:
        ap.error("--particles must be at least 2")
    pos4, vel4 = two_disks(a.particles, seed=a.seed, eps=a.eps,
                           mass_ratio=a.mass_ratio, impact=a.impact,
                           separation=a.separation, approach=a.approach,
                           inclination_deg=a.inclination,
                           core_frac=a.core_frac, core_a=a.core_a)
    formats.write_ic(a.out, pos4, vel4)
    print(f"wrote {pos4.shape[0]} particles to {a.out} "
          f"({pos4.nbytes + vel4.nbytes + 4} bytes)")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
