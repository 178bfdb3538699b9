"""The C++ drop-in builds without a GPU: the programs written against the
reference's API (tests/cpp) compile with g++ against include/ and link
against libkrans_cuda.so, which exports every entry point they call. Running
them is the GPU test (test_gpu_cpp_dropin.py)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("name", ["quickstart_cuda.cpp", "adapter_semantics.cpp"])
def test_cpp_dropin_compiles_and_links(tmp_path, name):
    lib = os.path.join(ROOT, "krans_b200")
    if not os.path.exists(os.path.join(lib, "libkrans_cuda.so")):
        pytest.skip("libkrans_cuda.so not built")
    exe = str(tmp_path / name.replace(".cpp", ""))
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-I", os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "tests", "cpp", name), "-o", exe, "-L", lib, "-lkrans_cuda",
                        f"-Wl,-rpath,{lib}"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]
    assert os.path.exists(exe)
