"""The benchmark's JSON contract, on the CPU: the keys of every line, the reference arm's line
(the oracle timed on the host cores, here on a sample of a few hundred photons), and the
reference arm's other ranks, which exit without work."""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402

BASE_KEYS = {"metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
             "vs_baseline", "dtype", "data", "config"}


def test_ordinal() -> None:
    assert [bench.ordinal(k) for k in (1, 2, 3, 4, 11, 12, 13, 21, 22, 23, 101, 111, 112)] == [
        "1st", "2nd", "3rd", "4th", "11th", "12th", "13th", "21st", "22nd", "23rd", "101st", "111th", "112th"]


def test_line_carries_the_base_keys() -> None:
    args = argparse.Namespace(steps=3, warmup=3)
    line = bench._line("m", 2.0, "rays/s", args, 5.0, {"workload": "w"}, e2e={"value": 1.0}, gpu_launches=6)
    assert BASE_KEYS <= set(line)
    assert line["steps"] == 3 and line["warmup"] == 3 and line["ms_per_step"] == 5.0
    assert line["higher_is_better"] is True and line["scaling"] == "weak" and line["vs_baseline"] is None
    assert line["e2e"] == {"value": 1.0} and line["gpu_launches"] == 6
    json.dumps(line)


def test_reference_arm_line(monkeypatch, capsys) -> None:
    """The reference arm on a sample of about 200 photons per step: one JSON line with the
    contract's keys, the cpu_baseline describing the run, and an e2e of the same value with no
    host-device copies."""
    pytest.importorskip("torch")
    monkeypatch.delenv("RANK", raising=False)
    monkeypatch.setattr(bench, "calibrate_stride", lambda specs, target_s: sum(s.n_rays for s in specs) // 200)
    bench.run_reference(argparse.Namespace(gpus=1, steps=2, warmup=3))
    lines = [ln for ln in capsys.readouterr().out.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert BASE_KEYS <= set(line) and line["impl"] == "reference"
    assert line["metric"] == bench.METRIC and line["unit"] == "rays/s" and line["value"] > 0
    assert line["steps"] == 2 and line["warmup"] == 3 and line["n_gpus"] == 1
    assert 150 <= line["config"]["photons_per_step"] <= 250
    cpu = line["cpu_baseline"]
    assert cpu["kind"] == "port" and cpu["value"] == line["value"] and cpu["cores"] >= 1 and cpu["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": "rays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_without_work() -> None:
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    p = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1",
                        "--warmup", "3"], cwd=ROOT, env=env, capture_output=True, text=True, timeout=120)
    assert p.returncode == 0 and p.stdout.strip() == ""
