"""The reference arm of bench.py on the host cores: it runs the oracle
port of the reference's CPU path and prints the one-line JSON contract."""
import json
import os
import subprocess
import sys

from conftest import ROOT


def test_reference_arm_prints_the_contract_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--steps", "1", "--warmup", "1", "--ref-points", "2"],
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["unit"] == "pts/s" and line["value"] > 0 and line["higher_is_better"]
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["value"] == line["value"]
    assert "ZK7" in line["config"]["workload"]


def test_kalman_reference_arm_prints_the_contract_line():
    for extra in ([], ["--kf-decoupled"]):
        out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--workload",
                              "kalman", "--impl", "reference", "--kf-dims", "3,16,16,1",
                              "--steps", "1", "--warmup", "1"] + extra,
                             capture_output=True, text=True, timeout=600, cwd=ROOT)
        assert out.returncode == 0, out.stderr[-2000:]
        line = json.loads(out.stdout.strip().splitlines()[-1])
        assert line["impl"] == "reference" and line["unit"] == "updates/s" and line["value"] > 0
        assert line["cpu_baseline"]["kind"] == "port" and line["e2e"]["value"] == line["value"]
        assert ("decoupled" in line["metric"]) == bool(extra)
        assert "EKF" in line["config"]["workload"]
