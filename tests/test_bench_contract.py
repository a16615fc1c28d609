"""The bench's reference arm runs on the host alone: its one JSON line keeps
the contract keys (metric, value, unit, impl, cpu_baseline, e2e) for the
workload the GPU arm measures, on a small sample."""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT


def test_reference_arm_json_line():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    if not os.path.exists(oracle.ref_exe("c2")):
        pytest.skip("compiled reference not built (no reference sources here)")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "3", "--ref-procs", "2"],
                         cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["unit"] == "particle-steps/s" and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] == 2
    assert d["cpu_baseline"]["cpu"]
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["config"]["particles"] == 65536 and d["config"]["mesh"] == 512
    # the GPU arm prints the same config object and takes the same warm-up
    sys.path.insert(0, ROOT)
    import bench
    assert d["config"] == bench.workload_config("medium")
    assert d["warmup"] == 3 and d["steps"] == 1


def test_reference_arm_served_is_unavailable():
    """The reference has no serving mode: --workload served prints its
    `unavailable` line and exits 0."""
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload",
                          "served", "--steps", "1", "--warmup", "3"],
                         cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    d = json.loads([l for l in out.stdout.splitlines() if l.startswith("{")][0])
    assert d["impl"] == "reference" and "serving" in d["unavailable"]


def test_reference_arm_other_ranks_exit_without_work():
    """Under torchrun only rank 0 times the reference; another rank prints
    nothing and exits 0 at once."""
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                          "--steps", "1", "--warmup", "3"],
                         cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    assert not [l for l in out.stdout.splitlines() if l.startswith("{")]
