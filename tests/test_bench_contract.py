"""CPU: the reference arm of bench.py (`--impl reference`) prints the same
metric, unit, direction and workload as the GPU arm's line, with the keys the
benchmark contract asks for: impl, cpu_baseline (kind, cores, sample, value)
and an e2e object with no host-device bytes. It times the reference library
compiled from its own sources (oracle/_ref) on the host cores."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libplsparse_ref.so")


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference library not built")
def test_reference_arm_line():
    sys.path.insert(0, ROOT)
    import bench

    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "1"],
                       capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads([l for l in r.stdout.splitlines() if l.startswith("{")][-1])
    assert line["impl"] == "reference"
    assert line["metric"] == bench.METRIC
    assert line["unit"] == "GB/s" and line["higher_is_better"] is True
    assert line["config"]["workload"].startswith("C2 power-law SpMV n=4194304 nnz=67061018")
    assert line["value"] > 0 and line["steps"] == 1
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == line["value"]
    assert "sample" in cb
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["h2d_bytes_per_step"] == 0
    assert e2e["d2h_bytes_per_step"] == 0


def test_reference_arm_other_ranks_exit_without_work():
    """Under torchrun the reference arm runs on rank 0 alone: any other rank
    exits 0 at once and prints no result line."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "1"],
                       capture_output=True, text=True, timeout=300, cwd=ROOT, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    assert not [l for l in r.stdout.splitlines() if l.startswith("{")]
