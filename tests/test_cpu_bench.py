"""bench.py's reference arm runs on the CPU only, so its JSON contract is
checked here on a tiny sample: same metric, unit and config as the GPU arm,
plus the keys of the reference arm. The replica path of the GPU arm (per-rank
seeds, max of device times and sum of counts over ranks) is checked with two
gloo ranks."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    sys.path.insert(0, ROOT)
    import bench
    # seed 3, batch 4, one step: one sampled instance per host core, drawn from
    # the four instances of the batch
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "0", "--batch", "4", "--seed", "3"],
                         capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads([l for l in out.stdout.splitlines() if l.startswith("{")][-1])
    assert line["impl"] == "reference"
    assert line["metric"] == bench.METRIC and line["unit"] == "solves/s" and line["higher_is_better"] is True
    assert line["value"] > 0 and line["cpu_baseline"]["value"] == line["value"]
    assert line["cpu_baseline"]["kind"] == ("reference" if bench._ref_available() else "port")
    count = max(1, os.cpu_count() or 1)
    assert line["cpu_baseline"]["cores"] >= 1 and line["sampled"] == count and line["converged"] == count
    assert line["e2e"] == {"value": line["value"], "unit": "solves/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}

    class A:
        batch = 4
    assert line["config"] == bench.batched_config(A, 1)  # identical to the GPU arm's config


def test_reference_sample_and_rate():
    sys.path.insert(0, ROOT)
    import bench
    batches = bench.make_batches(3 + 5, 16, 9)
    s1, S = bench.reference_sample(batches, 3, 5, 9)
    s2, _ = bench.reference_sample(batches, 3, 5, 9)
    count = max(5, os.cpu_count() or 1)  # at least one instance per host core
    assert s1 == s2 and len(s1) == count and S == min(8, count)
    assert [x[0] for x in s1] == [3 + q % 5 for q in range(count)]
    assert [x[2] for x in s1] == [q % S for q in range(count)]
    for (st, i, j) in s1:  # the instance lies in its stratum of the step's batch
        order = sorted(range(16), key=lambda q: (batches[st][q].A.nnz, q))
        assert (j * 16) // S <= order.index(i) < ((j + 1) * 16) // S
    v, per = bench.stratified_rate([1.0, 3.0, 2.0, 4.0], [0, 0, 1, 1], 2, 8)
    assert per == {"0": 2.0, "1": 3.0} and abs(v - 8 / 2.5) < 1e-12


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


def test_serving_request_options():
    # the serving stream's per-generator options: planted-kernel requests in
    # FP64, the batched workload's in mixed precision, LOBPCG for incidence
    sys.path.insert(0, ROOT)
    import bench
    import krans_b200 as kb
    pool = bench.serving_pool(6, 1e4, 3e4, kmax=4)
    kinds = {}
    for inst, solver in pool:
        o = bench.serving_opts(kb, inst, solver, 1)
        kinds.setdefault((inst.name, solver), set()).add(
            type(o).__name__ if solver == "lobpcg" else int(o.precision))
    assert kinds[("planted", "cyclic")] == {0}
    assert all(v == {1} for (name, solver), v in kinds.items() if solver == "cyclic" and name != "planted")
    assert kinds[("incidence", "lobpcg")] == {"LOBPCGOptions"}
