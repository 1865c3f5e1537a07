"""GPU parity of the leapfrog integrator, energy diagnostic, run loop and the
device-pointer drop-ins.

* kick / drift (plain and hi/lo compensated) are bit-exact against the
  oracle's mirror of the same float operations;
* energy within 1e-6 relative of the FP64 oracle;
* a 20-step trajectory of the reference's fixture IC stays within 2e-6 of
  reference_nbody.py's float64 frames, and the run loop writes the reference
  formats (frames byte layout, energy CSV columns);
* the plain all-pairs workload (12,000 particles, dt 0.005, 2,000 steps,
  energy every 10 steps) keeps |dE/E| <= 2e-4 (the 0.02 % band).
"""
import ctypes
import os

import numpy as np
import pytest

from nbodyssey_b200 import _lib as L
from nbodyssey_b200 import api, formats, ic
from oracle import oracle as O

pytestmark = pytest.mark.gpu

EPS = 0.05


@pytest.mark.parametrize("force", ["naive", "bh"])
@pytest.mark.parametrize("compensated", [True, False])
def test_one_step_bit_exact(force, compensated):
    pos, vel = ic.two_disks(5000, seed=21)
    dt = 0.005
    prm = api.SimParams(dt=dt, epsilon=EPS, force=force, theta=0.5,
                        traverse="warp", compensated=compensated)
    with api.Simulation(pos, vel, prm) as sim:
        a0 = sim.compute_forces()
        sim.step(1)
        p1 = sim.positions()
        lo1 = sim.position_lo()
        v1 = sim.velocities()
        a1 = sim.compute_forces()   # a(x1), deterministic recompute
    h = np.float32(0.5) * np.float32(dt)
    vh = O.kick(vel, a0, h)
    ep, elo = O.drift(pos, None, vh, np.float32(dt), compensated)
    assert np.array_equal(p1, ep)
    if compensated:
        assert np.array_equal(lo1, elo)
    else:
        assert np.all(lo1 == 0)
    assert np.array_equal(v1, O.kick(vh, a1, h))


@pytest.mark.parametrize("n", [1000, 30_000])
def test_energy_vs_fp64(n):
    pos, vel = ic.two_disks(n, seed=22)
    with api.Simulation(pos, vel, api.SimParams(epsilon=EPS)) as sim:
        e, ke, pe = sim.energy()
        mom = sim.momentum()
    ref = O.energy_f64(pos, vel, EPS)
    assert abs(ke - ref[1]) <= 1e-12 * abs(ref[1])
    assert abs(pe - ref[2]) <= 1e-6 * abs(ref[2])
    assert abs(e - ref[0]) <= 1e-6 * abs(ref[0])
    np.testing.assert_allclose(mom, ref[3:], rtol=1e-10, atol=1e-12)


def test_trajectory_and_formats_vs_reference(golden_dir, tmp_path):
    g = np.load(os.path.join(golden_dir, "refnbody.npz"))
    prm = api.SimParams(dt=0.01, epsilon=EPS, force="naive")
    out = tmp_path / "frames"
    csv = tmp_path / "e.csv"
    with api.Simulation(g["pos4"], g["vel4"], prm) as sim:
        st = sim.run(20, dump_every=5, out_dir=str(out), energy_log=str(csv))
    assert st["frames"] == 4
    names = sorted(os.listdir(out))
    assert names == list(g["frame_names_float64"])
    for k, name in enumerate(names):
        mine = formats.read_frame(str(out / name))
        ref = np.frombuffer(g["frames_float64"][k].tobytes()[4:], np.float32).reshape(-1, 4)
        assert (out / name).stat().st_size == g["frames_float64"][k].size
        assert np.array_equal(mine[:, 3], ref[:, 3])
        assert np.abs(mine[:, :3] - ref[:, :3]).max() < 2e-6
    mine = formats.read_energy_csv(str(csv))
    ref_rows = g["csv_float64"].tobytes().decode().splitlines()
    assert open(csv).readline() == formats.ENERGY_HEADER
    assert len(mine) == len(ref_rows) - 1 == 5          # 0, 5, 10, 15, 20
    ref = np.array([[float(x) for x in r.split(",")] for r in ref_rows[1:]])
    assert np.array_equal(mine["step"], ref[:, 0])
    np.testing.assert_allclose(mine["energy"], ref[:, 2], rtol=2e-6)
    np.testing.assert_allclose(mine["kinetic"], ref[:, 3], rtol=2e-6)


def test_energy_drift_plain_workload(tmp_path):
    """12,000 particles (two disks of 6,000, m = 1/6000), eps 0.05,
    dt 0.005, 2,000 steps, a row every 10 steps: 201 rows, |dE/E| <= 2e-4."""
    pos, vel = ic.plain_config(12_000, seed=0)
    prm = api.SimParams(dt=0.005, epsilon=EPS, force="naive")
    csv = tmp_path / "e.csv"
    with api.Simulation(pos, vel, prm) as sim:
        st = sim.run(2000, dump_every=10, out_dir=None, energy_log=str(csv))
    rows = formats.read_energy_csv(str(csv))
    assert len(rows) == 201
    assert rows["step"][0] == 0 and rows["step"][-1] == 2000
    assert np.abs(rows["rel_error"]).max() <= 2e-4
    assert abs(st["rel_final"]) <= 2e-4


@pytest.mark.parametrize("n,traverse", [(20_000, "warp"), (300_000, "thread")])
def test_graph_and_eager_identical(n, traverse):
    """The captured step graph and the eager launches (kernel by kernel, the
    Barnes-Hut chain with programmatic dependent launch) give the same bits;
    300,000 particles build three levels above the leaf groups."""
    pos, vel = ic.two_disks(n, seed=23)
    states = []
    for graphs in (True, False):
        prm = api.SimParams(dt=0.005, epsilon=EPS, force="bh", traverse=traverse)
        with api.Simulation(pos, vel, prm) as sim:
            sim.set_graphs(graphs)
            sim.step(5)
            states.append((sim.positions(), sim.velocities(), sim.position_lo()))
    for a, b in zip(*states):
        assert np.array_equal(a, b)


def test_timing_and_phases():
    pos, vel = ic.two_disks(50_000, seed=24)
    prm = api.SimParams(dt=0.005, epsilon=EPS, force="bh", traverse="warp")
    with api.Simulation(pos, vel, prm) as sim:
        sim.set_timing(True)
        sim.step(3)
        ph, calls = sim.phase_times()
        ms, fcalls = sim.force_timing()
    assert calls == 4 and fcalls == 4        # a(x0) + 3 steps
    assert all(ph[k] > 0 for k in ("prep", "morton", "sort", "build", "com", "walk"))
    assert ms > 0


def test_device_pointer_dropins():
    torch = pytest.importorskip("torch")
    lib = L.load()
    pos, vel = ic.two_disks(8000, seed=25)
    dpos = torch.from_numpy(pos).cuda()
    dvel = torch.from_numpy(vel).cuda()
    dacc = torch.zeros_like(dpos)
    ws = ctypes.c_void_p()
    L.check(lib.nb_workspace_create(ctypes.byref(ws)))
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    try:
        for force in ("naive", "bh"):
            prm = api.SimParams(dt=0.005, epsilon=EPS, force=force,
                                traverse="warp", compensated=False)
            pc = prm.to_c()
            L.check(lib.nb_compute_forces_dev(ws, 8000, ctypes.c_void_p(dpos.data_ptr()),
                                              ctypes.c_void_p(dacc.data_ptr()),
                                              ctypes.byref(pc), stream))
            torch.cuda.synchronize()
            with api.Simulation(pos, vel, prm) as sim:
                ref = sim.compute_forces()
                assert np.array_equal(dacc.cpu().numpy(), ref)
                # one reference-style leapfrog step on caller-owned buffers
                p2, v2, a2 = dpos.clone(), dvel.clone(), dacc.clone()
                L.check(lib.nb_leapfrog_step_dev(
                    ws, 8000, ctypes.c_void_p(p2.data_ptr()),
                    ctypes.c_void_p(v2.data_ptr()), ctypes.c_void_p(a2.data_ptr()),
                    ctypes.byref(pc), stream))
                torch.cuda.synchronize()
                sim.step(1)
                assert np.array_equal(p2.cpu().numpy(), sim.positions())
                assert np.array_equal(v2.cpu().numpy(), sim.velocities())
                e3 = np.zeros(3)
                L.check(lib.nb_total_energy_dev(ws, 8000, ctypes.c_void_p(p2.data_ptr()),
                                                ctypes.c_void_p(v2.data_ptr()),
                                                ctypes.byref(pc), L.ptr(e3), stream))
                assert np.array_equal(e3, np.array(sim.energy()))
    finally:
        lib.nb_workspace_destroy(ws)


def test_invalid_params_on_live_sim():
    pos, vel = ic.two_disks(100, seed=26)
    with api.Simulation(pos, vel, api.SimParams()) as sim:
        with pytest.raises(L.NbError) as ei:
            sim.set_params(api.SimParams(epsilon=0.0))
        assert ei.value.code == L.NB_ERR_INVALID
        sim.step(1)
        sim.sync()


@pytest.mark.parametrize("force", ["bh", "naive"])
def test_step_host_equals_upload_step_download(force):
    """nb_step_host (positions back on a second stream during the build and
    walk) gives the same state as nb_set_state_acc + nb_step + downloads."""
    pos, vel = ic.two_disks(30_000 if force == "bh" else 4_000, seed=51)
    prm = api.SimParams(dt=0.005, epsilon=0.05, theta=0.5, force=force,
                        traverse="warp")
    with api.Simulation(pos, vel, prm) as sim:
        acc = sim.compute_forces()
        p, v, a = pos, vel, acc
        for _ in range(3):
            p, v, a = sim.step_host(p, v, a)
    with api.Simulation(pos, vel, prm) as ref:
        ra = ref.compute_forces()
        rp, rv = pos, vel
        for _ in range(3):
            ref.set_state_acc(rp, rv, ra)
            ref.step(1)
            rp, rv, ra = ref.positions(), ref.velocities(), ref.accelerations()
    assert np.array_equal(p, rp) and np.array_equal(v, rv) and np.array_equal(a, ra)


@pytest.mark.parametrize("force", ["bh", "naive"])
def test_step_host_state_follows_the_device_trajectory(force):
    """nb_step_host_state with each call's output handed back: the same
    trajectory as nb_step on device-resident state, bit for bit (a(x) and the
    low-order position parts carry on on the device); positions changed by
    the caller start over as nb_set_state + nb_step."""
    pos, vel = ic.two_disks(30_000 if force == "bh" else 4_000, seed=52)
    prm = api.SimParams(dt=0.005, epsilon=0.05, theta=0.5, force=force,
                        traverse="warp")
    with api.Simulation(pos, vel, prm) as sim:
        p, v = pos, vel
        for _ in range(4):
            p, v = sim.step_host_state(p, v)
        # the caller moves one particle: a fresh start from that state
        p2 = p.copy()
        p2[7, 0] += 0.25
        q, w = sim.step_host_state(p2, v)
    with api.Simulation(pos, vel, prm) as ref:
        ref.step(4)
        rp, rv = ref.positions(), ref.velocities()
        assert np.array_equal(p, rp) and np.array_equal(v, rv)
        ref.set_state(p2, v)
        ref.step(1)
        assert np.array_equal(q, ref.positions()) and np.array_equal(w, ref.velocities())
