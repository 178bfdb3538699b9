"""GPU parity of the standalone SpMV / SpM^T V (krans_spmv_ex, the
MatrixInterface::multiply / multiply_transpose of the reference's
EigenSparseMatrixAdapter, include/krans/adapters/eigen/EigenSparseMatrixAdapter.hpp:34-57).

The UNIFORM and ROWTILE kernels sum each row in storage order with one
rounded product and one rounded addition per entry, so FP64 results must equal
the oracle's sequential CSR loop bit for bit, and FP32 results must equal the
same loop run in float32. The LANES kernel (warp butterfly) is checked to the
rounding bound instead. Edge cases: empty matrices, empty rows, rows longer
than one 2048-entry tile, every rows_per_block class, uniform rows of 1, 2
and 4 entries."""
import numpy as np
import pytest
import scipy.sparse as sp

from conftest import load_golden_matrix

pytestmark = pytest.mark.gpu


def seq_spmv(A, x, dtype):
    """Row sums in storage order in `dtype` (one rounding per product and per
    addition), vectorised over rows and sequential over positions."""
    A = A.tocsr()
    rp = A.indptr
    lens = np.diff(rp)
    s = np.zeros(A.shape[0], dtype)
    xv = x.astype(dtype)
    vals = A.data.astype(dtype)
    for j in range(int(lens.max()) if lens.size else 0):
        rows = np.flatnonzero(lens > j)
        k = rp[rows] + j
        s[rows] = s[rows] + vals[k] * xv[A.indices[k]]
    return s.astype(np.float64)


def matrices():
    from krans_b200 import generators as G
    r = np.random.default_rng(7)
    out = {
        "shift": G.shift_operator(3000, 5, 0.7, kernel=False).A,          # 2 per row (uniform)
        "incidence": G.graph_incidence(20000, 4, 8.0, seed=3, kernel=False).A,
        "planted": G.planted_kernel(3000, 2000, 8, seed=2, kernel=False).A,
        "mat2": load_golden_matrix(2)[0],
    }
    # one entry per row and four per row (uniform kernels of width 1 and 4)
    n = 5000
    out["diag"] = sp.csr_matrix((r.standard_normal(n), (np.arange(n), r.integers(0, 700, n))), shape=(n, 700))
    rows4 = np.repeat(np.arange(n), 4)
    cols4 = np.sort(np.argsort(r.random((n, 900)), axis=1)[:, :4], axis=1).ravel()
    out["four"] = sp.csr_matrix((r.standard_normal(4 * n), (rows4, cols4)), shape=(n, 900))
    # ragged: empty rows, a row of 9000 entries (spans five tiles), long tail
    lens = r.integers(0, 30, 3000)
    lens[::7] = 0
    lens[1234] = 9000
    rp = np.concatenate([[0], np.cumsum(lens)])
    ci = r.integers(0, 40000, int(rp[-1]))
    out["ragged"] = sp.csr_matrix((r.standard_normal(int(rp[-1])), ci, rp), shape=(3000, 40000))
    for A in out.values():
        A.sum_duplicates()  # canonical (sorted, unique columns): the oracle's storage order
    return out


@pytest.mark.parametrize("name", ["shift", "incidence", "planted", "mat2", "diag", "four", "ragged"])
def test_spmv_bit_identical_to_oracle(ctx, oracle, name):
    import krans_b200 as kb
    from krans_b200 import _capi as K
    A = matrices()[name]
    O = oracle.Csr.from_scipy(A)
    M = kb.CudaCsrMatrixAdapter.from_scipy(ctx, A, fp32=True)
    rng = np.random.default_rng(1)
    for trans in (0, 1):
        rows, cols = (A.shape[1], A.shape[0]) if trans else A.shape
        Aop = A.T.tocsr() if trans else A
        xh = rng.standard_normal(cols)
        x, y = kb.CudaVectorAdapter.from_numpy(ctx, xh), kb.CudaVectorAdapter(ctx, rows)
        mul = M.multiply_transpose if trans else M.multiply
        want64 = O.matvec(xh, trans=bool(trans))
        np.testing.assert_array_equal(want64, seq_spmv(Aop, xh, np.float64))
        want32 = seq_spmv(Aop, xh, np.float32)
        ulen = np.diff(Aop.indptr)
        kernels = [(K.KRANS_SPMV_AUTO, 0)] + [(K.KRANS_SPMV_ROWTILE, rb) for rb in (0, 1, 100, 256, 700, 2048)]
        if ulen.size and ulen.min() == ulen.max() and ulen[0] in (1, 2, 4):
            kernels.append((K.KRANS_SPMV_UNIFORM, 0))
        for kern, rb in kernels:
            M.set_spmv_tuning(trans, kern, rb)
            assert M.spmv_tuning(trans) == (kern, rb)
            y.set_zero()
            mul(x, y)
            np.testing.assert_array_equal(y.data(), want64, err_msg=f"{name} trans={trans} kernel={kern} rb={rb}")
            mul(x, y, precision=kb.Precision.MIXED)
            np.testing.assert_array_equal(y.data(), want32, err_msg=f"f32 {name} trans={trans} kernel={kern}")
        M.set_spmv_tuning(trans, K.KRANS_SPMV_AUTO, 0, x_evict_last=True)  # cache policy only
        mul(x, y)
        np.testing.assert_array_equal(y.data(), want64)
        M.set_spmv_tuning(trans, K.KRANS_SPMV_LANES)
        mul(x, y)
        bound = 64 * 2.2e-16 * (abs(Aop) @ np.abs(xh))
        assert np.all(np.abs(y.data() - want64) <= bound + 1e-300)
        M.set_spmv_tuning(trans, K.KRANS_SPMV_AUTO)


def test_spmv_empty_and_invalid(ctx):
    import krans_b200 as kb
    from krans_b200 import _capi as K
    A = sp.csr_matrix((0, 5))
    M = kb.CudaCsrMatrixAdapter.from_scipy(ctx, A)
    x, y = kb.CudaVectorAdapter(ctx, 5), kb.CudaVectorAdapter(ctx, 0)
    M.multiply(x, y)
    M.multiply_transpose(y, x)
    assert not np.any(x.data())
    Z = sp.csr_matrix((4, 3))  # no entries at all
    M = kb.CudaCsrMatrixAdapter.from_scipy(ctx, Z)
    x, y = kb.CudaVectorAdapter.from_numpy(ctx, np.ones(3)), kb.CudaVectorAdapter.from_numpy(ctx, np.ones(4))
    M.multiply(x, y)
    np.testing.assert_array_equal(y.data(), np.zeros(4))
    with pytest.raises(ValueError, match="UNIFORM"):
        M.set_spmv_tuning(False, K.KRANS_SPMV_UNIFORM)
    with pytest.raises(ValueError, match="rows_per_block"):
        M.set_spmv_tuning(False, K.KRANS_SPMV_ROWTILE, 5000)
    with pytest.raises(ValueError, match="unknown kernel"):
        M.set_spmv_tuning(False, 9)
    with pytest.raises(ValueError, match="FP32"):
        M.multiply(x, y, precision=kb.Precision.MIXED)
