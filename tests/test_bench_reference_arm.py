"""bench.py's reference arm (the FP64 C port of predict_auto + lr_refine on
the host cores) keeps the one-JSON-line contract without a GPU, and under a
multi-rank launch only rank 0 prints."""

import json
import os
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(env_extra):
    env = dict(os.environ)
    env.update(env_extra)
    p = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "1", "--cpu-seconds", "0.5"],
                       cwd=REPO, env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    return [ln for ln in p.stdout.splitlines() if ln.strip()]


@pytest.mark.timeout(900)
def test_reference_arm_prints_one_contract_line():
    lines = _run({"RANK": "0", "WORLD_SIZE": "1", "LOCAL_RANK": "0"})
    assert len(lines) == 1
    res = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
                "cpu_baseline", "e2e"):
        assert key in res, key
    assert res["impl"] == "reference"
    assert res["value"] > 0 and res["higher_is_better"] is True
    assert res["cpu_baseline"]["kind"] == "port" and res["cpu_baseline"]["cores"] >= 1
    assert res["cpu_baseline"]["value"] == res["value"]
    assert res["e2e"] == {"value": res["value"], "unit": res["unit"],
                          "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert "workload" in res["config"]


@pytest.mark.timeout(300)
def test_reference_arm_other_ranks_exit_quietly():
    assert _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}) == []
