"""Build libkrans_cuda.so in-tree with nvcc for sm_100a (B200).

    python -m krans_b200.build [--force]

Compiles every krans_b200/csrc/*.cu and *.cpp into one shared library next
to this file. No GPU is needed (nvcc cross-compiles).
"""
from __future__ import annotations

import argparse
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.environ.get("KRANS_B200_BUILD_LIB", os.path.join(HERE, "libkrans_cuda.so"))
BUILD_DIR = os.environ.get("KRANS_B200_BUILD_DIR", os.path.join(HERE, "_build"))
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", "nvcc")
# extra nvcc flags for tuning builds (e.g. "-DKR_SPMV_ROWS=8")
EXTRA = os.environ.get("KRANS_NVCC_FLAGS", "").split()


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _deps():
    return _sources() + sorted(glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
                               + glob.glob(os.path.join(HERE, "..", "include", "*.h"))
                               + glob.glob(os.path.join(HERE, "..", "include", "krans", "**", "*.hpp"),
                                           recursive=True)
                               + [os.path.join(HERE, "cli", "krans_nullspace.cpp")])


def up_to_date() -> bool:
    if not os.path.exists(LIB) or not os.path.exists(os.path.join(os.path.dirname(LIB), "krans_nullspace")):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(p) <= t for p in _deps())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(BUILD_DIR, exist_ok=True)
    objs = []
    procs = []
    for src in _sources():
        obj = os.path.join(BUILD_DIR, os.path.basename(src) + ".o")
        cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
               "--extended-lambda", "-Xcompiler", "-fPIC,-O3", *EXTRA, "-c", src, "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
        objs.append(obj)
    failed = False
    for src, p in procs:
        out, _ = p.communicate()
        if out.strip() and (verbose or p.returncode != 0):
            sys.stderr.write(f"--- {os.path.basename(src)}\n{out}")
        if p.returncode != 0:
            failed = True
    if failed:
        raise RuntimeError("nvcc failed (see output above)")
    tmp = LIB + ".tmp"
    subprocess.run([NVCC, *ARCH, "-shared", "--cudart", "static", "-o", tmp, *objs], check=True)
    os.replace(tmp, LIB)
    build_cli()
    return LIB


CLI_SRC = os.path.join(HERE, "cli", "krans_nullspace.cpp")
CLI = os.path.join(os.path.dirname(LIB), "krans_nullspace")


def build_cli() -> str:
    """The command-line tool (C++ over the drop-in headers and the library)."""
    libdir = os.path.dirname(LIB)
    tmp = CLI + ".tmp"
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(HERE, "..", "include"), CLI_SRC, "-o", tmp,
                    "-L", libdir, "-l:" + os.path.basename(LIB), "-Wl,-rpath,$ORIGIN"], check=True)
    os.replace(tmp, CLI)
    return CLI


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
