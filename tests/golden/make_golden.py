"""Regenerate the committed golden fixtures under tests/golden/.

Run in the development container (it reads the reference checkout and needs
g++); GPU test runs only read the committed outputs:

    python tests/golden/make_golden.py /path/to/reference

Outputs
  rng_normals.txt   exact doubles (C99 hex) of std::mt19937(seed) +
                    std::normal_distribution<double>(0,1) under libstdc++,
                    from gen_rng_golden.cpp: the generator behind the
                    reference's StdVectorFactory/EigenVectorFactory.
  matN.npz          the reference's test matrices data/matN.ija (N=1..6),
                    parsed as the IJA loader does (3 header integers m n nnz,
                    then 0-based "i j v" triplets, duplicates summed,
                    src/IO/MatrixLoader.cpp:21-56), stored as CSR
                    (int32 indptr/indices, float64 data).
"""
import os
import subprocess
import sys
import tempfile

import numpy as np
import scipy.sparse as sp

HERE = os.path.dirname(os.path.abspath(__file__))

# nullities of the reference's fixtures (tests/test_cyclic_lanczos.cpp:192,313-314,
# benchmarks/workers/verification_suite.cpp:135-140)
NULLITY = {1: 5, 2: 15, 3: 10, 4: 15, 5: 20, 6: 25}


def load_ija(path):
    with open(path) as f:
        tok = f.read().split()
    m, n, nnz = int(tok[0]), int(tok[1]), int(tok[2])
    body = np.array(tok[3:], dtype=object).reshape(-1, 3)
    i = body[:, 0].astype(np.int64)
    j = body[:, 1].astype(np.int64)
    v = body[:, 2].astype(np.float64)
    A = sp.coo_matrix((v, (i, j)), shape=(m, n)).tocsr()  # sums duplicates
    A.sum_duplicates()
    A.sort_indices()
    return A, nnz, len(v)


def main(ref):
    with tempfile.TemporaryDirectory() as td:
        exe = os.path.join(td, "gen_rng")
        subprocess.run(["g++", "-O2", "-o", exe, os.path.join(HERE, "gen_rng_golden.cpp")],
                       check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    with open(os.path.join(HERE, "rng_normals.txt"), "w") as f:
        f.write(out)
    for k, nul in NULLITY.items():
        A, hdr_nnz, read = load_ija(os.path.join(ref, "data", f"mat{k}.ija"))
        np.savez_compressed(os.path.join(HERE, f"mat{k}.npz"), m=A.shape[0], n=A.shape[1],
                            indptr=A.indptr.astype(np.int32), indices=A.indices.astype(np.int32),
                            data=A.data, nullity=nul, header_nnz=hdr_nnz, triplets=read)
        print(f"mat{k}: {A.shape} nnz={A.nnz} nullity={nul}")


if __name__ == "__main__":
    ref_root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("KRANS_REFERENCE_ROOT")
    if not ref_root:
        sys.exit("usage: make_golden.py REFERENCE_ROOT (or set KRANS_REFERENCE_ROOT): the root of a "
                 "Deep-SANE/krans checkout, whose data/mat*.ija files are read")
    main(ref_root)
