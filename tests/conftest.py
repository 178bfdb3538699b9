import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA engine)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    return O


def load_golden_matrix(k):
    import scipy.sparse as sp
    z = np.load(os.path.join(GOLDEN, f"mat{k}.npz"))
    A = sp.csr_matrix((z["data"], z["indices"], z["indptr"]), shape=(int(z["m"]), int(z["n"])))
    return A, int(z["nullity"])


@pytest.fixture(scope="session")
def ctx():
    import krans_b200 as kb
    return kb.Context(0)


def dense_kernel(A, k):
    """Orthonormal rows spanning the k smallest right singular vectors."""
    _, s, Vt = np.linalg.svd(A.toarray())
    return Vt[-k:]
