"""The bench's reference arm on CPU: the JSON line it prints for the Born
workload on a machine without a GPU, where the reference's own CUDA Born
drivers cannot run and the oracle port stands in on the host cores (with a
GPU the arm times those drivers, on a record cut to the length their 32-bit
history index admits)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_cpu_port_line():
    env = dict(os.environ, OMP_NUM_THREADS=str(min(os.cpu_count() or 1, 8)))
    p = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0"],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    line = [x for x in p.stdout.splitlines() if x.startswith("{")][-1]
    d = json.loads(line)
    assert d["impl"] == "reference"
    assert d["metric"] == "Gcells/s" and d["unit"] == "Gcell-updates/s" and d["higher_is_better"] is True
    assert d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert "no CUDA device" in d["reference_gpu"]["unavailable"]


def test_reference_arm_names_why_the_learned_workloads_have_no_reference():
    for wl in ("fwi_learned", "cnn_train", "fwi_1000x3400"):
        p = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", wl, "--steps", "1",
                            "--warmup", "0"], cwd=ROOT, capture_output=True, text=True, timeout=300)
        assert p.returncode == 0, p.stderr[-2000:]
        d = json.loads([x for x in p.stdout.splitlines() if x.startswith("{")][-1])
        assert d["impl"] == "reference" and d["unavailable"]


def test_cnn_step_flops():
    sys.path.insert(0, ROOT)
    import bench
    chans = [16, 32, 32, 16]
    per = [2 * 9 * 16 * 32, 2 * 9 * 32 * 32, 2 * 9 * 32 * 16]
    # forward of every layer + weight gradient of every layer + data gradient of all but the first
    assert bench.cnn_step_flops(chans, 10) == 10 * (2 * sum(per) + per[1] + per[2])
