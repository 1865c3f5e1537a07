"""scripts/gpu_bench.sh's protocol on this library (nbodyssey_b200.gpu_bench,
quick mode): the theta = 0 gates of both tree walks pass (mean < 1e-4), the
sweep reports ms/call for every (N, method) up to 100,000, the energy runs
write their logs.  When the reference's galaxy_sim built for sm_100a is
present (oracle/_ref/galaxy_sim, built by oracle/build_ref.sh), it runs
beside on the same ic.bin files: its gates pass too and its ms/call is
recorded next to ours."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "galaxy_sim")


def test_gpu_bench_quick(tmp_path):
    cmd = [sys.executable, "-m", "nbodyssey_b200.gpu_bench", "--quick",
           "--out", str(tmp_path)]
    if os.path.exists(REF):
        cmd += ["--ref-bin", REF]
    r = subprocess.run(cmd, cwd=str(tmp_path), capture_output=True, text=True,
                       timeout=1800, env=dict(os.environ, PYTHONPATH=ROOT))
    assert r.returncode == 0, r.stderr[-3000:]
    s = json.load(open(str(tmp_path / "summary.json")))
    for k, v in s["gates"].items():
        if "theta0" in k and "theta0.5" not in k:
            assert v["mean"] < 1e-4, (k, v)
    assert len(s["sweep"]) == 4 * 3 + 2 * 2
    for row in s["sweep"]:
        assert row["ours_ms_per_call"] > 0
        if os.path.exists(REF):
            assert row["ref_ms_per_call"] > 0
    assert abs(s["energy"]["ours_naive"]) < 2e-4
    print(json.dumps(s["sweep"]))
