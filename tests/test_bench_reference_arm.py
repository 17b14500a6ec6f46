"""bench.py --impl reference on the host CPU: one JSON line with the contract's keys, the same
workload config as the GPU arm (its own step length in `step`), and under torchrun only rank 0
prints."""
import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SMALL = ["--impl", "reference", "--cells", "20000", "--steps", "2", "--warmup", "1", "--cpu-sample-iters", "1"]


def json_lines(out):
    return [json.loads(l) for l in out.splitlines() if l.startswith("{")]


def test_reference_arm_prints_one_contract_line():
    r = subprocess.run([sys.executable, "bench.py"] + SMALL, cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = json_lines(r.stdout)
    assert len(lines) == 1
    d = lines[0]
    assert d["impl"] == "reference"
    assert d["metric"] == d["unit"] == "cell-updates/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 2 and d["warmup"] == 1 and d["n_gpus"] == 1
    assert d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["kind"] == "port"
    assert d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    c = d["config"]
    assert c["cells"] == c["dims"][0] * c["dims"][1] * c["dims"][2]
    assert 0.8 * 20000 < c["cells"] < 1.2 * 20000
    assert c["workload"].startswith("fighter plain solve, ") and c["fixed_states"] == "cycle at 0 m"
    assert "iterations_per_step" not in c  # the step length is each arm's own: its `step` key
    assert d["step"]["iterations"] == 1  # what the arm timed per step (--cpu-sample-iters)


def test_reference_arm_under_torchrun_prints_on_rank_zero_only():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--gpus", "2"] + SMALL
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = json_lines(r.stdout)
    assert len(lines) == 1 and lines[0]["impl"] == "reference" and lines[0]["n_gpus"] == 2


def test_roofline_traffic_comes_from_the_kernels_profile_summary():
    """roofline.traffic is the committed range capture of the default kernel (DRAM bytes per cell
    and stage over whole stages) times the cells; a kernel without a summary reports none."""
    import bench
    n = 4131324
    assert bench.measured_traffic("k_stage_pair", n) == 52.6 * n
    assert bench.measured_traffic("k_stage_tma", n) == 35.8 * n
    assert bench.measured_traffic("k_stage_cell", n) is None
    assert bench.KERNEL_NAMES[4] == "k_stage_pair"
