"""The `galaxy_sim` command line (src/main.cu:18-215) on the B200 library.

    python -m nbodyssey_b200.galaxy_sim --ic ic.bin [--steps N] [--dt f]
        [--eps f] [--G f] [--dump-every N] [--out dir] [--energy-log csv]
        [--force naive|bh] [--theta f] [--traverse thread|warp]
        [--compare-forces]

Flags and defaults follow src/main.cu:18-70 (dt 0.01, eps 0.05, G 1, theta
0.5, naive, thread, 1000 steps, a frame + energy row every 5 steps, frames to
./frames, energy log benchmarks/energy_gpu.csv).  Extra flags: --key-bits
(30|63), --plain-drift (no hi/lo compensation), --walk (pair|list|dfs),
--checkpoint PATH (a state file of the final state: the ic.bin layout plus a
trailer with the parameters, the low-order position parts and a(x)) and
--resume PATH (continue from such a file, with its parameters, bit for bit as
if the run had not stopped; --ic is then not needed).  The run loop itself is
native (nb_run): frames stream out asynchronously while the next steps run.
"""
from __future__ import annotations

import argparse
import sys

from . import _lib as L
from . import api, formats


def parse_args(argv=None):
    ap = argparse.ArgumentParser(prog="galaxy_sim", description=__doc__,
                                 formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--ic")
    ap.add_argument("--out", default="frames")
    ap.add_argument("--energy-log", default="benchmarks/energy_gpu.csv")
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--dump-every", type=int, default=5)
    ap.add_argument("--dt", type=float, default=0.01)
    ap.add_argument("--eps", type=float, default=0.05)
    ap.add_argument("--G", type=float, default=1.0)
    ap.add_argument("--theta", type=float, default=0.5)
    ap.add_argument("--force", choices=["naive", "bh", "auto"], default="naive")
    ap.add_argument("--traverse", choices=["thread", "warp"], default="thread")
    ap.add_argument("--compare-forces", action="store_true")
    ap.add_argument("--key-bits", type=int, choices=[30, 63], default=30)
    ap.add_argument("--plain-drift", action="store_true")
    ap.add_argument("--walk", choices=["pair", "list", "dfs"], default="pair")
    ap.add_argument("--checkpoint", help="write the final state to this state file")
    ap.add_argument("--resume", help="start from this state file instead of --ic")
    a = ap.parse_args(argv)
    if not a.ic and not a.resume:
        ap.error("one of --ic or --resume is required")
    return a


def main(argv=None):
    a = parse_args(argv)
    params = api.SimParams(dt=a.dt, epsilon=a.eps, G=a.G, theta=a.theta,
                           force=a.force, traverse=a.traverse, key_bits=a.key_bits,
                           compensated=not a.plain_drift, walk_kernel=a.walk)
    try:
        if a.resume:
            sim = api.Simulation.from_state(a.resume)
            params = sim.params
            a.dt, a.eps, a.theta = params.dt, params.epsilon, params.theta
            a.force, a.traverse = params.force, params.traverse
        else:
            pos4, vel4 = formats.read_ic(a.ic)
            sim = api.Simulation(pos4, vel4, params)
    except (OSError, formats.FormatError, L.NbError) as e:
        print(e, file=sys.stderr)
        return 1
    n = sim.n
    with sim:
        if a.compare_forces:
            # src/main.cu:75-112; gpu_bench.sh greps the second line
            mx, mean = sim.compare_forces()
            print("naive vs barnes-hut, theta=%.3g, traverse=%s, n=%d" %
                  (a.theta, a.traverse, n))
            print("relative force error: max %.3e, mean %.3e" % (mx, mean))
            return 0
        bh = a.force == "bh"
        e0, ke0, pe0 = sim.energy()
        head = "n=%d dt=%.4g eps=%.4g steps=%d force=%s" % (
            n, a.dt, a.eps, a.steps, "barnes-hut" if bh else "naive")
        if bh:
            head += " theta=%.3g traverse=%s" % (a.theta, a.traverse)
        print(head)
        print("E0=%.6e KE0=%.6e PE0=%.6e" % (e0, ke0, pe0))
        st = sim.run(a.steps, a.dump_every, a.out, a.energy_log, timing=True)
        ms, calls = st["force_ms"], st["force_calls"]
        print("force pipeline: %d calls, %.1f ms total, %.3f ms/call" %
              (calls, ms, ms / max(calls, 1)))
        if bh:
            total = sum(v for k, v in st["phase_ms"].items() if k != "energy")
            print("barnes-hut pipeline, per-call average over %d calls:" % calls)
            for k in ("prep", "morton", "sort", "build", "com", "walk"):
                v = st["phase_ms"][k]
                print("  %-9s %8.3f ms  (%4.1f%%)" % (k, v, 100.0 * v / total if total else 0))
        else:
            gips = float(n) * n * calls / (ms * 1e-3) / 1e9 if ms > 0 else 0.0
            print("throughput: %.2f Ginteractions/s (~%.1f GFLOP/s at 20 flop/pair)" %
                  (gips, gips * 20.0))
        print("wrote %d frames to %s" % (st["frames"], a.out))
        if a.checkpoint:
            sim.save_state(a.checkpoint)
            print("wrote state to %s" % a.checkpoint)
    return 0


if __name__ == "__main__":
    sys.exit(main())
