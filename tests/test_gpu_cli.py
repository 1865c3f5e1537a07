"""The galaxy_sim command line on the GPU: flags and defaults of src/main.cu,
frames and energy rows in the reference formats, and the --compare-forces
line scripts/gpu_bench.sh greps (theta 0 gate: mean < 1e-4)."""
import os
import re
import subprocess
import sys

import numpy as np
import pytest

from nbodyssey_b200 import formats, ic

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(args, cwd):
    return subprocess.run([sys.executable, "-m", "nbodyssey_b200.galaxy_sim"] + args,
                          cwd=cwd, capture_output=True, text=True, timeout=600,
                          env=dict(os.environ, PYTHONPATH=ROOT))


@pytest.mark.parametrize("force", ["naive", "bh"])
def test_run_writes_frames_and_energy(tmp_path, force):
    pos, vel = ic.two_disks(3000, seed=40)
    icp = tmp_path / "ic.bin"
    formats.write_ic(str(icp), pos, vel)
    r = _run(["--ic", str(icp), "--steps", "20", "--dump-every", "5", "--dt", "0.005",
              "--out", str(tmp_path / "frames"), "--energy-log", str(tmp_path / "e.csv"),
              "--force", force, "--traverse", "warp"], tmp_path)
    assert r.returncode == 0, r.stderr
    assert "force pipeline:" in r.stdout and "wrote 4 frames" in r.stdout
    names = sorted(os.listdir(tmp_path / "frames"))
    assert names == ["frame_%05d.bin" % k for k in range(4)]
    fr = formats.read_frame(str(tmp_path / "frames" / names[-1]))
    assert fr.shape == (3000, 4) and np.array_equal(fr[:, 3], pos[:, 3])
    rows = formats.read_energy_csv(str(tmp_path / "e.csv"))
    assert list(rows["step"]) == [0, 5, 10, 15, 20]
    assert np.abs(rows["rel_error"]).max() < 1e-3


def test_compare_forces_line(tmp_path):
    pos, vel = ic.two_disks(5000, seed=41)
    icp = tmp_path / "ic.bin"
    formats.write_ic(str(icp), pos, vel)
    for tv in ("thread", "warp"):
        r = _run(["--ic", str(icp), "--compare-forces", "--theta", "0",
                  "--traverse", tv], tmp_path)
        assert r.returncode == 0, r.stderr
        m = re.search(r"relative force error: max (\S+), mean (\S+)", r.stdout)
        assert m and float(m.group(2)) < 1e-4


def test_bad_ic_is_an_error(tmp_path):
    bad = tmp_path / "bad.bin"
    bad.write_bytes(b"\x05\x00\x00\x00" + b"\x00" * 40)
    r = _run(["--ic", str(bad)], tmp_path)
    assert r.returncode != 0 and "truncated" in r.stderr


def test_checkpoint_and_resume(tmp_path):
    """--checkpoint after 20 steps, --resume for 20 more: the final state
    equals 40 uninterrupted steps bit for bit."""
    pos, vel = ic.two_disks(3000, seed=42)
    icp = tmp_path / "ic.bin"
    formats.write_ic(str(icp), pos, vel)
    common = ["--dump-every", "20", "--dt", "0.005", "--force", "bh", "--traverse", "warp",
              "--energy-log", str(tmp_path / "e.csv")]
    r = _run(["--ic", str(icp), "--steps", "40", "--out", str(tmp_path / "a"),
              "--checkpoint", str(tmp_path / "full.bin")] + common, tmp_path)
    assert r.returncode == 0, r.stderr
    r = _run(["--ic", str(icp), "--steps", "20", "--out", str(tmp_path / "b"),
              "--checkpoint", str(tmp_path / "half.bin")] + common, tmp_path)
    assert r.returncode == 0, r.stderr
    r = _run(["--resume", str(tmp_path / "half.bin"), "--steps", "20",
              "--out", str(tmp_path / "c"), "--checkpoint", str(tmp_path / "end.bin"),
              "--dump-every", "20", "--energy-log", str(tmp_path / "e2.csv")], tmp_path)
    assert r.returncode == 0, r.stderr
    a = open(str(tmp_path / "full.bin"), "rb").read()
    b = open(str(tmp_path / "end.bin"), "rb").read()
    assert a == b
