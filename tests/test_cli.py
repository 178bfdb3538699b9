"""The command-line tool krans_b200/krans_nullspace (the reference's
apps/krans_nullspace.cpp for its iterative solvers): flags, exit codes and
outputs (N.csv: one row per entry, one column per vector, 17 digits;
report.json with rank, nullity, timings, residuals, max off-diagonal dot)."""
import json
import os
import subprocess

import numpy as np
import pytest

from conftest import load_golden_matrix

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "krans_b200", "krans_nullspace")


def run(*args, cwd=None):
    return subprocess.run([CLI, *args], capture_output=True, text=True, timeout=600, cwd=cwd)


def test_cli_usage_and_argument_errors(tmp_path):
    from krans_b200 import build
    build.build()
    assert os.path.exists(CLI)
    r = run("--help")
    assert r.returncode == 0 and "--solver" in r.stderr
    assert run("--solver", "cyclic").returncode == 2                     # --input is required
    r = run("--solver", "svd", "--input", "x.mtx")
    assert r.returncode == 2 and "Unknown solver" in r.stderr
    assert run("--bogus").returncode == 2
    assert run("--solver", "cyclic", "--input", "x.mtx", "--device", "cpu").returncode == 2


def _write_ija(path, A):
    C = A.tocoo()
    with open(path, "w") as f:
        f.write(f"{A.shape[0]} {A.shape[1]} {C.nnz}\n")
        for i, j, v in zip(C.row, C.col, C.data):
            f.write(f"{int(i)} {int(j)} {float(v)!r}\n")


@pytest.mark.gpu
@pytest.mark.parametrize("solver", ["cyclic", "lobpcg"])
def test_cli_golden_matrix(tmp_path, solver):
    A, nul = load_golden_matrix(1)
    p = tmp_path / "mat1.ija"
    _write_ija(p, A)
    args = ["--solver", solver, "--input", str(p), "--k", str(nul), "--out", str(tmp_path / "N.csv"),
            "--report", str(tmp_path / "report.json")]
    if solver == "lobpcg":
        args += ["--lobpcg-block", "8"]
    r = run(*args, cwd=str(tmp_path))
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith(f"OK [{solver}]")
    N = np.loadtxt(tmp_path / "N.csv", delimiter=",", ndmin=2)
    assert N.shape == (A.shape[1], nul)
    assert np.max(np.linalg.norm(A @ N, axis=0)) <= 1e-8
    rep = json.load(open(tmp_path / "report.json"))
    assert rep["solver"] == solver and rep["rows"] == A.shape[0] and rep["cols"] == A.shape[1]
    assert rep["nullity"] == nul and rep["rank"] == A.shape[1] - nul
    assert len(rep["residuals"]) == nul and max(rep["residuals"]) <= 1e-8
    assert rep["max_offdiag_abs_dot"] <= 1e-8
    assert set(rep["timings_ms"]) == {"load", "solve"}
