#!/usr/bin/env python3
"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs only where the nbodyssey sources are present (pass their path with
--reference, required).  It imports the reference's Python
oracles -- scripts/lbvh_check.py, scripts/reference_nbody.py,
scripts/barnes_hut_reference.py, scripts/generate_ic.py -- calls their
functions unmodified, runs reference_nbody.py as a program, and stores the
inputs and outputs as small .npz files.  Tests never read the reference; they
read these fixtures.

Fixtures:
  lbvh_seed1.npz    lbvh_check.py's own test case (seed-1 blobs + 24
                    coincident points, n=3024), positions cast to float32:
                    63-bit keys, stable order, Karras topology, FP64 centres of
                    mass and sizes, thread walks of 192 targets and warp walks
                    of 8 warps at theta 0 and 0.5.  The 30-bit topology is
                    lbvh_check.build_tree applied to the 30-bit keys shifted to
                    the top of a 64-bit word (an order-preserving change of the
                    delta values, so the tree is the 30-bit Karras tree).
  refnbody.npz      a 512-particle generate_ic disk pair; reference_nbody.py
                    run for 20 steps (dump every 5) in float32 and float64:
                    ic.bin bytes, every frame's bytes, the energy CSV text,
                    plus accelerations / total_energy at t=0.
  bh_octree.npz     barnes_hut_reference.sweep statistics (n=2000, 200
                    targets) for theta in {0, 0.3, 0.5, 0.7}.
"""
import argparse
import io
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def lbvh_fixture(lbvh):
    rng = np.random.default_rng(1)
    a = rng.normal([-2.0, 0.0, 0.0], 0.7, size=(1500, 3))
    b = rng.normal([2.0, 0.5, 0.1], 0.7, size=(1500, 3))
    dupes = np.tile([[0.123, -0.456, 0.789]], (24, 1))
    pos = np.concatenate([a, b, dupes]).astype(np.float32)
    n = pos.shape[0]
    mass32 = np.full(n, 1.0 / n, dtype=np.float32)
    eps2 = lbvh.EPS * lbvh.EPS

    keys = lbvh.morton_keys(pos)                     # float32 in, NEP 50
    order = sorted(range(n), key=lambda i: keys[i])
    keys_sorted = [keys[i] for i in order]
    pos_sorted = pos[order].astype(np.float64)
    mass_sorted = mass32[order].astype(np.float64)
    children, parent = lbvh.build_tree(keys_sorted)
    lbvh.check_topology(children, parent, n)
    com, size = lbvh.compute_com(children, pos_sorted, mass_sorted, n)

    # 30-bit keys are the top 30 bits of the 63-bit keys (the quantisation
    # scale differs by 2^11, an exact power of two).
    keys30 = [k >> 33 for k in keys]
    order30 = sorted(range(n), key=lambda i: keys30[i])
    ks30 = [keys30[i] for i in order30]
    children30, parent30 = lbvh.build_tree([k << 34 for k in ks30])
    lbvh.check_topology(children30, parent30, n)

    sample = rng.choice(n, size=192, replace=False)
    out = {}
    for th in (0.0, 0.5):
        accs, inters, depths = [], [], []
        for t in sample:
            acc, ni, depth = lbvh.traverse(int(t), pos_sorted, mass_sorted,
                                           children, com, size, n, th, eps2)
            accs.append(acc)
            inters.append(ni)
            depths.append(depth)
        tag = "t%02d" % int(round(th * 10))
        out["thread_acc_" + tag] = np.array(accs)
        out["thread_inter_" + tag] = np.array(inters, np.int64)
        out["thread_depth_" + tag] = np.array(depths, np.int32)
    warp_ids = rng.choice(n // 32, size=8, replace=False)
    for th in (0.0, 0.5):
        accs, inters = [], []
        for w in warp_ids:
            a_w, lanes, ni, depth = lbvh.traverse_warp(
                int(w) * 32, pos_sorted, mass_sorted, children, com, size, n,
                th, eps2)
            accs.append(a_w)
            inters.append(ni)
        tag = "t%02d" % int(round(th * 10))
        out["warp_acc_" + tag] = np.array(accs)
        out["warp_inter_" + tag] = np.array(inters, np.int64)
    exact = lbvh.exact_accel(sample, pos_sorted, mass_sorted, eps2)

    np.savez_compressed(
        os.path.join(HERE, "lbvh_seed1.npz"),
        pos=pos, mass=mass32, eps=np.float64(lbvh.EPS),
        keys63=np.array(keys, np.uint64), order63=np.array(order, np.int64),
        children63=np.array(children, np.int32),
        parent63=np.array(parent, np.int32),
        com=np.asarray(com, np.float64), size=np.asarray(size, np.float64),
        keys30=np.array(keys30, np.uint64), order30=np.array(order30, np.int64),
        children30=np.array(children30, np.int32),
        parent30=np.array(parent30, np.int32),
        sample=np.asarray(sample, np.int64),
        warp_ids=np.asarray(warp_ids, np.int64), exact=exact, **out)
    print("lbvh_seed1.npz: n=%d, dup keys=%d" % (n, n - len(set(keys))))


def refnbody_fixture(ref_dir, gen, ref):
    rng = np.random.default_rng(7)
    pa, va = gen.build_disk(256, 1.0, 1.0, [-3.0, -0.5, 0.0], [0.3, 0.0, 0.0],
                            0.0, 1.0, 0.05, rng)
    pb, vb = gen.build_disk(256, 1.0, 1.0, [3.0, 0.5, 0.0], [-0.3, 0.0, 0.0],
                            np.radians(30.0), -1.0, 0.05, rng)
    pos4 = np.concatenate([pa, pb])
    vel4 = np.concatenate([va, vb])
    res = {}
    with tempfile.TemporaryDirectory() as td:
        icp = os.path.join(td, "ic.bin")
        gen.write_ic(icp, pos4, vel4)
        with open(icp, "rb") as f:
            res["ic_bytes"] = np.frombuffer(f.read(), np.uint8)
        for dt_name in ("float32", "float64"):
            od = os.path.join(td, "frames_" + dt_name)
            el = os.path.join(td, "energy_%s.csv" % dt_name)
            subprocess.run([sys.executable,
                            os.path.join(ref_dir, "scripts", "reference_nbody.py"),
                            "--ic", icp, "--steps", "20", "--dump-every", "5",
                            "--dt", "0.01", "--eps", "0.05", "--out", od,
                            "--energy-log", el, "--dtype", dt_name],
                           check=True, stdout=subprocess.DEVNULL)
            frames = sorted(os.listdir(od))
            res["frame_names_" + dt_name] = np.array(frames)
            res["frames_" + dt_name] = np.stack(
                [np.frombuffer(open(os.path.join(od, fr), "rb").read(), np.uint8)
                 for fr in frames])
            res["csv_" + dt_name] = np.frombuffer(open(el, "rb").read(), np.uint8)
    pos = pos4[:, :3]
    mass = pos4[:, 3]
    eps2 = np.float32(0.05 * 0.05)
    res["acc_f32"] = ref.accelerations(pos.astype(np.float32),
                                       mass.astype(np.float32), eps2,
                                       np.float32(1.0), 2048, np.float32)
    res["acc_f64"] = ref.accelerations(pos.astype(np.float64),
                                       mass.astype(np.float64),
                                       np.float64(0.05 * 0.05), np.float64(1.0),
                                       2048, np.float64)
    res["energy0"] = np.array(ref.total_energy(pos, vel4[:, :3], mass,
                                               np.float64(0.05 * 0.05), 1.0, 2048))
    np.savez_compressed(os.path.join(HERE, "refnbody.npz"), pos4=pos4,
                        vel4=vel4, **res)
    print("refnbody.npz: n=%d" % pos4.shape[0])


def octree_fixture(gen, bhr):
    rng = np.random.default_rng(3)
    pa, _ = gen.build_disk(1000, 1.0, 1.0, [-4.0, 0.0, 0.0], [0, 0, 0], 0.0,
                           1.0, 0.05, rng)
    pb, _ = gen.build_disk(1000, 1.0, 1.0, [4.0, 1.0, 0.0], [0, 0, 0],
                           np.radians(30.0), -1.0, 0.05, rng)
    pos4 = np.concatenate([pa, pb])
    thetas = np.array([0.0, 0.3, 0.5, 0.7])
    srng = np.random.default_rng(11)
    med, inter = bhr.sweep(pos4[:, :3].astype(np.float64),
                           pos4[:, 3].astype(np.float64), 0.05 * 0.05, thetas,
                           200, srng)
    np.savez_compressed(os.path.join(HERE, "bh_octree.npz"), pos4=pos4,
                        thetas=thetas, med_err=med, mean_inter=inter)
    print("bh_octree.npz: med err", med, "inter", inter)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True,
                    help="checkout of the nbodyssey reference")
    args = ap.parse_args()
    sys.path.insert(0, os.path.join(args.reference, "scripts"))
    import barnes_hut_reference as bhr
    import generate_ic as gen
    import lbvh_check as lbvh
    import reference_nbody as ref

    lbvh_fixture(lbvh)
    refnbody_fixture(args.reference, gen, ref)
    octree_fixture(gen, bhr)


if __name__ == "__main__":
    main()
