"""The GPU benchmark protocol of the reference (scripts/gpu_bench.sh:37-71) on
this library, optionally with the reference's own `galaxy_sim` timed beside
it on the same initial conditions.

    python -m nbodyssey_b200.gpu_bench [--ref-bin PATH] [--out DIR] [--quick]

Steps, as the reference's script takes them:

1. correctness gates (gpu_bench.sh:37-48): theta = 0 must reproduce the naive
   forces for both tree walks, `--compare-forces` mean relative error < 1e-4
   (N = 20,000); theta = 0.5 reported;
2. sweep (gpu_bench.sh:51-56): N in {4096, 12000, 50000, 100000, 200000,
   400000, 1000000} x {naive, bh-thread, bh-warp} at theta 0.5, 10 steps,
   `ms/call` of the force pipeline as printed by the CLI;
3. theta sensitivity (gpu_bench.sh:59-62): theta 0.3 and 0.8 at N = 100,000;
4. energy (gpu_bench.sh:65-71): N = 12,000, 1,500 steps, a row every 100
   steps, naive and Barnes-Hut warp, final relative energy error.

Initial conditions come from this package's two-disk generator (seeded),
written as ic.bin, so the reference binary reads the same files.  Every run
goes through the `galaxy_sim` command line of each side.  Results: a CSV
`n,method,theta,ms_per_call,ref_ms_per_call` (the reference's
gpu_results.csv plus the reference column) and a JSON summary in --out.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import tempfile

from . import formats, ic

SIZES = (4096, 12000, 50000, 100000, 200000, 400000, 1000000)
METHODS = (("naive", ["--force", "naive"]),
           ("bh-thread", ["--force", "bh", "--traverse", "thread"]),
           ("bh-warp", ["--force", "bh", "--traverse", "warp"]))


def _ours():
    return [sys.executable, "-m", "nbodyssey_b200.galaxy_sim"]


_LOG_DIR = None


def _run(cmd, timeout=1800, log=None):
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    if _LOG_DIR and log:   # per-run logs, as gpu_bench.sh keeps in benchmarks/logs
        with open(os.path.join(_LOG_DIR, log + ".txt"), "w") as f:
            f.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
    if r.returncode != 0:
        raise RuntimeError("%s failed (%d): %s" % (" ".join(cmd), r.returncode,
                                                    r.stderr[-2000:]))
    return r.stdout


def ms_per_call(stdout):
    """The force pipeline's ms/call (the field gpu_bench.sh's awk takes)."""
    m = re.search(r"force pipeline: .*?([0-9.eE+-]+) ms/call", stdout)
    return float(m.group(1)) if m else None


def compare_mean(stdout):
    m = re.search(r"relative force error: max (\S+), mean (\S+)", stdout)
    return (float(m.group(1)), float(m.group(2))) if m else (None, None)


def final_rel_energy(csv_path):
    rows = formats.read_energy_csv(csv_path)
    return float(rows["rel_error"][-1])


def main(argv=None):
    ap = argparse.ArgumentParser(prog="gpu_bench", description=__doc__,
                                 formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--ref-bin", help="the reference's galaxy_sim built for this GPU")
    ap.add_argument("--out", default="gpu_bench_out")
    ap.add_argument("--quick", action="store_true",
                    help="sizes up to 100,000 and 150 energy steps (a smoke run)")
    a = ap.parse_args(argv)
    os.makedirs(a.out, exist_ok=True)
    global _LOG_DIR
    _LOG_DIR = os.path.join(a.out, "logs")
    os.makedirs(_LOG_DIR, exist_ok=True)
    scratch = tempfile.mkdtemp(prefix="nb_gpu_bench_")
    sides = [("ours", _ours())]
    if a.ref_bin:
        sides.append(("ref", [os.path.abspath(a.ref_bin)]))
    sizes = [n for n in SIZES if not a.quick or n <= 100000]
    summary = {"gates": {}, "sweep": [], "energy": {}}

    def icfile(n):
        path = os.path.join(scratch, "ic_%d.bin" % n)
        if not os.path.exists(path):
            pos, vel = ic.two_disks(n, seed=0)
            formats.write_ic(path, pos, vel)
        return path

    def case(cmd, n, th, extra, log, steps=10):
        return _run(cmd + ["--ic", icfile(n), "--steps", str(steps),
                           "--dump-every", "1000000", "--out",
                           os.path.join(scratch, "frames"), "--energy-log",
                           os.path.join(scratch, "e.csv"), "--theta", str(th)] + extra,
                    log=log)

    # 1. gates
    for name, cmd in sides:
        for tv in ("thread", "warp"):
            for th in (0.0, 0.5):
                out = _run(cmd + ["--ic", icfile(20000), "--compare-forces", "--theta",
                                  str(th), "--traverse", tv],
                           log="%s_gate_theta%g_%s" % (name, th, tv))
                mx, mean = compare_mean(out)
                summary["gates"]["%s_%s_theta%g" % (name, tv, th)] = {"max": mx, "mean": mean}
                if th == 0.0 and not (mean is not None and mean < 1e-4):
                    raise SystemExit("GATE FAILED (%s, %s): theta=0 mean error %s" %
                                     (name, tv, mean))
    # 2. + 3. sweep
    rows = []
    plan = [(n, lab, 0.5, extra) for n in sizes for lab, extra in METHODS]
    plan += [(100000, lab, th, extra) for th in (0.3, 0.8) for lab, extra in METHODS[1:]]
    for n, lab, th, extra in plan:
        row = {"n": n, "method": lab, "theta": th}
        for name, cmd in sides:
            row["%s_ms_per_call" % name] = ms_per_call(
                case(cmd, n, th, extra, "%s_%s_n%d_theta%g" % (name, lab, n, th)))
        rows.append(row)
        print(json.dumps(row), flush=True)
    summary["sweep"] = rows
    with open(os.path.join(a.out, "gpu_results.csv"), "w") as f:
        f.write("n,method,theta,ms_per_call,ref_ms_per_call\n")
        for r in rows:
            ref = r.get("ref_ms_per_call")
            f.write("%d,%s,%g,%.3f,%s\n" % (r["n"], r["method"], r["theta"],
                                            r["ours_ms_per_call"],
                                            "%.3f" % ref if ref is not None else ""))
    # 4. energy
    steps = 150 if a.quick else 1500
    for name, cmd in sides:
        for lab, extra in (("naive", ["--force", "naive"]),
                           ("bh", ["--force", "bh", "--theta", "0.5", "--traverse", "warp"])):
            csv = os.path.join(a.out, "energy_%s_%s.csv" % (name, lab))
            _run(cmd + ["--ic", icfile(12000), "--steps", str(steps), "--dump-every", "100",
                        "--out", os.path.join(scratch, "frames_e"),
                        "--energy-log", csv] + extra, log="%s_energy_%s" % (name, lab))
            summary["energy"]["%s_%s" % (name, lab)] = final_rel_energy(csv)
    with open(os.path.join(a.out, "summary.json"), "w") as f:
        json.dump(summary, f, indent=1)
    print(json.dumps(summary["energy"]))
    return 0


if __name__ == "__main__":
    sys.exit(main())
