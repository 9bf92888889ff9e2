"""bench.py --impl reference on the CPU: it runs alone (no CUDA library is
loaded), prints one JSON line with the contract's keys and the same config
keys as the GPU arm, and its solve reaches the tolerance."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_small_grid():
    env = dict(os.environ, WORLD_SIZE="1", RANK="0", LOCAL_RANK="0")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--grid", "24", "--steps", "2", "--warmup", "1"],
                         capture_output=True, text=True, env=env, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1, out.stdout
    d = json.loads(lines[0])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["higher_is_better"] is False
    assert d["config"]["rows"] == 24 ** 3 and d["config"]["nv"] == 8
    assert set(d["config"]) == {"workload", "rows", "nnz", "nv", "rhs_per_gpu_per_step",
                                "tolerance", "l2"}
    assert d["cpu_baseline"]["kind"] in ("reference", "port")
    assert d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["true_rel_residual"] <= 1e-8
    assert d["steps"] == 2 and d["value"] > 0
