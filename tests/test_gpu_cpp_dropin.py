"""The C++ drop-in: programs written against the reference's API (the
quickstart with CudaCsrMatrixAdapter + CudaVectorFactory, and the adapter
semantics) compiled with g++ against include/ and libkrans_cuda.so."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
pytestmark = pytest.mark.gpu


def build_and_run(src, tmp_path):
    exe = str(tmp_path / os.path.basename(src).replace(".cpp", ""))
    lib = os.path.join(ROOT, "krans_b200")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), src, "-o", exe,
                    "-L", lib, "-lkrans_cuda", f"-Wl,-rpath,{lib}"], check=True)
    return subprocess.run([exe], capture_output=True, text=True, timeout=300)


def test_quickstart_with_cuda_adapters(tmp_path):
    r = build_and_run(os.path.join(ROOT, "tests", "cpp", "quickstart_cuda.cpp"), tmp_path)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = [l for l in r.stdout.splitlines() if l.startswith(("cyclic", "lobpcg"))]
    assert len(lines) == 2 and all(l.split()[1] == "3" for l in lines)


def test_adapter_semantics(tmp_path):
    r = build_and_run(os.path.join(ROOT, "tests", "cpp", "adapter_semantics.cpp"), tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "adapter semantics OK" in r.stdout
