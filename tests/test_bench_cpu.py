"""The reference arm of bench.py on the host cores: it runs the oracle
port of the reference's CPU path and prints the one-line JSON contract."""
import json
import os
import subprocess
import sys

from conftest import ROOT


def test_reference_arm_prints_the_contract_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--steps", "1", "--warmup", "1"],
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["unit"] == "pts/s" and line["value"] > 0 and line["higher_is_better"]
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["value"] == line["value"]
    assert "ZK7" in line["config"]["workload"]
    # every thread carries the same share of the sample
    assert "32 per thread" in line["cpu_baseline"]["sample"]


def test_gpus_flag_relaunches_one_rank_per_gpu():
    """bench.py --gpus N started without a launcher re-runs itself as N
    ranks under torch.distributed.run, rendezvous on the loopback address."""
    sys.path.insert(0, ROOT)
    import bench

    cmd = bench.relaunch_cmd(4, ["--gpus", "4", "--steps", "3"], 29511)
    assert cmd[1:4] == ["-m", "torch.distributed.run", "--nnodes=1"]
    assert "--nproc-per-node=4" in cmd and "--master-addr=127.0.0.1" in cmd
    assert "--master-port=29511" in cmd
    assert cmd[-5:] == [os.path.join(ROOT, "bench.py"), "--gpus", "4", "--steps", "3"]
    # a launcher whose world size disagrees with --gpus is refused
    env = dict(os.environ, WORLD_SIZE="2", RANK="0", LOCAL_RANK="0")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "4"],
                         capture_output=True, text=True, timeout=300, cwd=ROOT, env=env)
    assert out.returncode == 2 and "WORLD_SIZE=2" in out.stderr


def test_ngd_reference_arm_prints_the_contract_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--workload", "ngd",
                          "--impl", "reference", "--steps", "1", "--warmup", "1"],
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "steps/s" and line["value"] > 0
    assert "heat" in line["config"]["workload"] and line["cpu_baseline"]["kind"] == "port"


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


def test_autotuner_summary_of_the_report():
    """The bench line's autotuner field from the library's report rows
    (kernel, D0, K, |A|, width, precision, chosen id, trial times): the ZK7
    shapes by variant name without repeats, the others counted, a pin named."""
    sys.path.insert(0, ROOT)
    import bench
    from dnnf90_b200 import api

    rows = [("bell_adj", 4, 7, 330, 128, "f32", 3, [1.0, 0.5]),
            ("bell_adj", 4, 7, 330, 128, "f32", 3, [1.0, 0.5]),   # a second ZK7 net
            ("bell_fwd_train", 4, 7, 330, 128, "f64", 2, [2.0, 1.0]),
            ("bell_fwd_train", 3, 4, 35, 256, "f32", 2, [1.0, 2.0]),
            ("bell_adj", 3, 4, 35, 256, "f32", 1, [1.0, 0.9]),
            ("bell_adj", 2, 5, 21, 64, "f32", 1, [1.0, 0.9])]

    class Stub:
        FWD_VARIANTS = api.FWD_VARIANTS
        ADJ_VARIANTS = api.ADJ_VARIANTS

        @staticmethod
        def tune_report():
            return rows

    out = bench.autotuner_summary(Stub)
    assert out["shapes"] == 6
    assert out["zk7"] == ["bell_adj f32: tiled", "bell_fwd_train f64: v8"]
    assert out["others"] == {"bell_adj f32 v5-shared": 2, "bell_fwd_train f32 v8": 1}
    assert "pinned" not in out
    assert bench.autotuner_summary(Stub, "3,3")["pinned"] == "3,3"
