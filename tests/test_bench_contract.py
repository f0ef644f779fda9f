"""bench.py's reference arm on CPU (small N): one JSON line with the contract's keys, the
same metric and config as the GPU arm builds for the same arguments, and an e2e equal to
its value (no host-device copies on the CPU)."""
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)


def test_reference_arm_line():
    out = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference",
                          "--n", "512", "--steps", "1", "--warmup", "0"],
                         capture_output=True, text=True, timeout=300, cwd=REPO)
    assert out.returncode == 0, out.stderr
    d = json.loads(out.stdout.strip().splitlines()[-1])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config", "impl",
              "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["unit"] == "solves/s" and d["higher_is_better"]
    assert d["value"] > 0 and d["e2e"]["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert "host" in d["cpu_baseline"]
    sys.path.insert(0, REPO)
    import bench
    saved = sys.argv
    sys.argv = ["bench.py", "--n", "512"]
    try:
        args = bench.parse()
    finally:
        sys.argv = saved
    assert d["metric"] == bench.dense_metric(512)
    assert d["config"] == bench.dense_config(args, 512, 1)
