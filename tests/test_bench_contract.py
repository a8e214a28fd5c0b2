"""bench.py's reference arm on the CPU (it times the C oracle on the host's cores, no GPU): the one JSON line the
driver reads, with every key of the contract, on the headline workload (the full PD14 microcircuit, drawn on the
host) with the GPU arm's config, and under a multi-rank launch nothing but rank 0's line."""

import json
import os
import pathlib
import subprocess
import sys

ROOT = pathlib.Path(__file__).resolve().parents[1]


def run_bench(*extra, env=None):
    e = dict(os.environ, **(env or {}))
    proc = subprocess.run([sys.executable, str(ROOT / "bench.py"), *extra], cwd=ROOT, env=e, capture_output=True,
                          text=True, timeout=600)
    assert proc.returncode == 0, proc.stderr[-2000:]
    return [json.loads(line) for line in proc.stdout.splitlines() if line.startswith("{")]


def test_reference_arm_prints_one_contract_line():
    lines = run_bench("--impl", "reference", "--steps", "1", "--warmup", "3")
    assert len(lines) == 1
    d = lines[0]
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
                "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["metric"] == "synaptic events/s" and d["unit"] == "events/s"
    assert d["higher_is_better"] is True and d["warmup"] >= 3 and d["value"] > 0
    assert d["config"]["workload"] == "pd14_config2" and d["config"]["neurons"] == 77169
    assert d["config"]["sim_steps_per_step"] == 1000 and d["config"]["window_steps"] == 1000
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_prints_nothing_on_other_ranks():
    assert run_bench("--impl", "reference", "--config", "1", "--steps", "1", "--warmup", "3",
                     env={"RANK": "1", "WORLD_SIZE": "2"}) == []


def test_reference_arm_config1():
    (d,) = run_bench("--impl", "reference", "--config", "1", "--steps", "1", "--warmup", "3")
    assert d["config"]["workload"] == "brunel_A_config1" and d["config"]["neurons"] == 12500
    assert d["value"] > 0 and d["impl"] == "reference"
