"""Energy drift of a workload against the force module's accuracy settings.

    python -m nbodyssey_b200.drift_study [--workload twodisk12k|precision262k]
        [--thetas 0.5,0.3,...] [--dts 0.005,0.0025] [--traverse warp|thread]
        [--json out.json]

Runs the workload for the same physical time (2,000 steps at its base dt)
with all-pairs and with Barnes-Hut at each opening angle and each timestep,
and reports per run the largest |E(t) - E0| / |E0| over 20 checkpoints, the
final momentum drift and the force evaluation's ms per call.  Comparing
timesteps separates integration error (shrinks with dt) from force-error
drift (follows theta, not dt); the reference's energy study
(docs/PERFORMANCE.md:94-104) reports only the end point of one setting.
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np

from . import api, ic

WORKLOADS = {
    # N, generator, eps, base dt, steps
    "twodisk12k": (12_000, ic.two_disks, 0.05, 0.005, 2000),
    "precision262k": (262_144, ic.precision_config, 0.01, 0.002, 2000),
}


def run_one(pos, vel, params, steps, checkpoints=20):
    with api.Simulation(pos, vel, params) as sim:
        e0 = sim.energy()[0]
        p0 = sim.momentum()
        worst = 0.0
        per = max(1, steps // checkpoints)
        done = 0
        while done < steps:
            k = min(per, steps - done)
            sim.step(k)
            done += k
            worst = max(worst, abs(sim.energy()[0] - e0) / abs(e0))
        dp = float(np.linalg.norm(sim.momentum() - p0))
        sim.set_timing(True)
        sim.reset_timing()
        sim.step(10)
        sim.sync()
        ms, calls = sim.force_timing()
    return {"max_rel_energy": worst, "momentum_drift": dp,
            "ms_per_force": ms / max(calls, 1)}


def main(argv=None):
    ap = argparse.ArgumentParser(prog="drift_study", description=__doc__,
                                 formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="twodisk12k")
    ap.add_argument("--thetas", default="0.5,0.4,0.3,0.2,0.15,0.1")
    ap.add_argument("--dts", default="", help="timesteps (default: the workload's, "
                                              "and half of it at the first theta)")
    ap.add_argument("--traverse", choices=["warp", "thread"], default="warp")
    ap.add_argument("--json")
    a = ap.parse_args(argv)
    n, gen, eps, dt0, steps0 = WORKLOADS[a.workload]
    pos, vel = gen(n, seed=0)
    thetas = [float(x) for x in a.thetas.split(",") if x]
    runs = [("naive", None, dt0)]
    runs += [("bh", th, dt0) for th in thetas]
    if a.dts:
        runs += [("bh", th, float(d)) for th in thetas for d in a.dts.split(",")
                 if float(d) != dt0]
    else:
        runs.append(("bh", thetas[0], dt0 / 2))
    out = []
    for force, th, dt in runs:
        steps = int(round(steps0 * dt0 / dt))
        prm = api.SimParams(dt=dt, epsilon=eps, force=force, theta=th or 0.5,
                            traverse=a.traverse)
        t0 = time.perf_counter()
        r = run_one(pos, vel, prm, steps)
        r.update({"workload": a.workload, "n": n, "force": force, "theta": th,
                  "traverse": a.traverse, "dt": dt, "steps": steps,
                  "wall_s": time.perf_counter() - t0})
        print(json.dumps(r), flush=True)
        out.append(r)
    if a.json:
        with open(a.json, "w") as f:
            json.dump(out, f, indent=1)
    return 0


if __name__ == "__main__":
    sys.exit(main())
