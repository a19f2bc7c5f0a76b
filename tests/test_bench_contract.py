"""bench.py's reference arm (the reference's own CUDA build, oracle/_ref/ref_run) prints one JSON
line with the keys the benchmark contract names; without a GPU it prints its `unavailable` line;
under a multi-rank launch only rank 0 works and prints."""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT

ARGS = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", "c1",
        "--steps", "2", "--warmup", "1"]


def _run(env_extra, args=ARGS):
    env = dict(os.environ, **env_extra)
    return subprocess.run(args, cwd=ROOT, env=env, capture_output=True, text=True, timeout=900)


def _cuda() -> bool:
    import torch
    return torch.cuda.is_available()


def test_reference_arm_without_a_gpu_prints_unavailable():
    if _cuda():
        pytest.skip("a GPU is present: the GPU test covers the reference arm")
    p = _run({"RANK": "0", "WORLD_SIZE": "1", "LOCAL_RANK": "0"})
    assert p.returncode == 0, p.stderr
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, p.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and "GPU" in d["unavailable"]


@pytest.mark.gpu
def test_reference_arm_prints_the_contract_line():
    p = _run({"RANK": "0", "WORLD_SIZE": "1", "LOCAL_RANK": "0"}, ARGS + ["--ref-samples", "20000"])
    assert p.returncode == 0, p.stderr
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, p.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "Gillespie transitions/s" and d["unit"] == "transitions/s"
    assert d["value"] > 0 and d["ms_per_step"] > 0
    assert (d["n_gpus"], d["steps"], d["warmup"]) == (1, 2, 1)
    assert d["higher_is_better"] is True and d["scaling"] == "weak" and d["vs_baseline"] is None
    assert d["dtype"] == "f32" and d["data"] == "synthetic"
    assert d["config"]["workload"].startswith("c1:") and d["config"]["trajectories"] == 20000
    assert d["config"]["transitions_per_step"] > 0
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["unit"] == d["unit"] and cb["kind"] == "reference"
    e2e = d["e2e"]
    assert 0 < e2e["value"] <= d["value"] * 1.01 and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_reference_arm_other_ranks_exit_without_work():
    p = _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert p.returncode == 0, p.stderr
    assert not [l for l in p.stdout.splitlines() if l.startswith("{")]
