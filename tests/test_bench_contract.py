"""bench.py's reference arm (the CPU restatement of the reference's PT-ICM
loop on the default line's jobs) runs without a GPU and prints the one JSON
line the benchmark contract asks of it: the GPU arm's metric, unit and
configuration, `impl: reference`, a cpu_baseline describing the run, and an
e2e block with no host-device copies."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_the_contract_line():
    cp = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "3",
                         "--cpu-stride", "256"], cwd=ROOT, capture_output=True, text=True, timeout=900)
    assert cp.returncode == 0, cp.stderr[-2000:]
    line = json.loads(cp.stdout.strip().splitlines()[-1])
    sys.path.insert(0, ROOT)
    import bench
    assert line["impl"] == "reference"
    assert line["metric"] == bench.METRIC and line["config"] == bench.C3_CONFIG  # the GPU arm's metric and config
    assert line["unit"] == "flips/s" and line["higher_is_better"] is True and line["value"] > 0
    assert line["n_gpus"] == 1 and line["steps"] == 1 and line["warmup"] == 3
    base = line["cpu_baseline"]
    assert base["kind"] == "port" and base["value"] == line["value"] and base["cores"] >= 1
    assert "1 of the 256 jobs" in base["sample"] and "5000 sweeps" in base["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": "flips/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    # the per-step time is the whole batch's flips at the measured rate
    assert abs(line["ms_per_step"] - bench.c3_flips(bench.c3_jobs()) / line["value"] * 1e3) < 1e-6 * line["ms_per_step"]


def test_reference_arm_under_torchrun_prints_one_line_from_rank_0():
    """Launched like the GPU arm on two ranks, the reference arm runs on rank
    0 alone and prints one line; the other rank exits 0 without work."""
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "3", "--cpu-stride", "256"]
    cp = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=900)
    assert cp.returncode == 0, cp.stderr[-2000:]
    lines = [ln for ln in cp.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
