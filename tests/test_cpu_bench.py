"""bench.py's reference arm runs the CPU oracle only, so its JSON contract is
checked here on a tiny sample: same metric, unit and config as the GPU arm,
plus the keys of the reference arm."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    sys.path.insert(0, ROOT)
    import bench
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "0", "--batch", "8", "--ref-sample", "1"],
                         capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads([l for l in out.stdout.splitlines() if l.startswith("{")][-1])
    assert line["impl"] == "reference"
    assert line["metric"] == bench.METRIC and line["unit"] == "solves/s" and line["higher_is_better"] is True
    assert line["value"] > 0 and line["cpu_baseline"]["value"] == line["value"]
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"] == {"value": line["value"], "unit": "solves/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["config"]["workload"] == bench.WORKLOAD


def test_indicator_kernel_distance():
    sys.path.insert(0, ROOT)
    import numpy as np
    import bench
    labels = np.array([0, 0, 1, 1, 1, 2])
    K = np.zeros((3, 6))
    for c in range(3):
        K[c, labels == c] = 1.0
        K[c] /= np.linalg.norm(K[c])
    Q = np.linalg.qr(np.random.default_rng(0).standard_normal((3, 3)))[0]
    assert bench.kernel_dist_indicator(Q @ K, labels, 3) < 1e-14
    V = Q @ K
    V[0] += 1e-3 * np.random.default_rng(1).standard_normal(6)
    V = np.linalg.qr(V.T)[0].T
    assert 1e-5 < bench.kernel_dist_indicator(V, labels, 3) < 1e-2
