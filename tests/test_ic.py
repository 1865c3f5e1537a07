"""The seeded IC generator and its ``ic.bin`` CLI (CPU only)."""
import numpy as np

from nbodyssey_b200 import formats, ic


def test_cli_writes_readable_ic(tmp_path, capsys):
    out = tmp_path / "ic.bin"
    assert ic.main(["--particles", "3001", "--out", str(out), "--seed", "4",
                    "--mass-ratio", "0.5"]) == 0
    assert "wrote 3001 particles" in capsys.readouterr().out
    assert out.stat().st_size == 4 + 3001 * 32
    pos, vel = formats.read_ic(str(out))
    p2, v2 = ic.two_disks(3001, seed=4, mass_ratio=0.5)
    assert np.array_equal(pos, p2) and np.array_equal(vel, v2)
    # equal particle masses up to the rounding of the split, total mass
    # 1 + mass_ratio
    assert np.allclose(pos[:, 3], pos[0, 3], rtol=1e-3)
    assert abs(pos[:, 3].astype(np.float64).sum() - 1.5) < 1e-4
    assert np.all(vel[:, 3] == 0.0)


def test_recipe_geometry():
    pos, vel = ic.two_disks(20_000, seed=1)
    n_a = 10_000
    ca = pos[:n_a, :3].astype(np.float64).mean(axis=0)
    cb = pos[n_a:, :3].astype(np.float64).mean(axis=0)
    assert np.allclose(ca, [-10.0, -2.0, 0.0], atol=0.1)
    assert np.allclose(cb, [10.0, 2.0, 0.0], atol=0.1)
    # disks truncated at R = 5 around their centres (A untilted)
    ra = np.hypot(pos[:n_a, 0] + 10.0, pos[:n_a, 1] + 2.0)
    assert ra.max() <= 5.0 + 1e-4
    # bulk velocities +-0.25 along x, net momentum zero for equal masses
    assert abs(vel[:n_a, 0].mean() - 0.25) < 0.02
    assert abs(vel[n_a:, 0].mean() + 0.25) < 0.02


def test_seeded_and_distinct():
    a = ic.two_disks(1000, seed=7)
    b = ic.two_disks(1000, seed=7)
    c = ic.two_disks(1000, seed=8)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert not np.array_equal(a[0], c[0])


def test_plummer_core_variant():
    pos, vel = ic.two_disks(4000, seed=2, eps=0.01, core_frac=0.1, core_a=0.1)
    assert pos.shape == (4000, 4) and np.isfinite(pos).all()
    assert np.isfinite(vel).all()
