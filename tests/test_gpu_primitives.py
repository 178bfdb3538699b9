"""GPU parity of the VectorInterface / MatrixInterface / VectorFactory
primitives (C-ABI, called through the Python host mirror) against numpy, the
CPU oracle and the libstdc++ golden RNG vectors."""
import os

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import GOLDEN, load_golden_matrix

pytestmark = pytest.mark.gpu


def test_vector_ops(ctx):
    import krans_b200 as kb
    rng = np.random.default_rng(0)
    for n in [0, 1, 7, 1000, 100_003]:
        a, b = rng.standard_normal(n), rng.standard_normal(n)
        va = kb.CudaVectorAdapter.from_numpy(ctx, a)
        vb = kb.CudaVectorAdapter.from_numpy(ctx, b)
        assert va.size() == n
        assert abs(va.dot(vb) - a @ b) <= 1e-12 * (1 + np.abs(a) @ np.abs(b))
        assert abs(va.norm() - np.linalg.norm(a)) <= 1e-13 * (1 + np.linalg.norm(a))
        va.add_scaled(vb, -0.75)  # device axpy may fuse the multiply-add (1 ulp)
        assert np.all(np.abs(va.data() - (a - 0.75 * b)) <= 2.3e-16 * (np.abs(a) + 0.75 * np.abs(b)))
        ref = va.data() * 3.0
        va.scale(3.0)
        np.testing.assert_array_equal(va.data(), ref)
        c = va.clone()
        np.testing.assert_array_equal(c.data(), va.data())
        c.set_zero()
        assert not np.any(c.data())
        c.copy_from(vb)
        np.testing.assert_array_equal(c.data(), b)
        c.normalize()
        if n:
            assert abs(np.linalg.norm(c.data()) - 1.0) < 1e-14
    z = kb.CudaVectorAdapter(ctx, 5)
    z.normalize()  # norm 0: unchanged (VectorInterface::normalize "if norm > 0")
    assert not np.any(z.data())
    with pytest.raises(ValueError):
        kb.CudaVectorAdapter(ctx, 3).dot(kb.CudaVectorAdapter(ctx, 4))
    with pytest.raises(ValueError):
        kb.CudaVectorAdapter(ctx, 3).add_scaled(np.zeros(3), 1.0)


@pytest.mark.parametrize("which", ["shift", "mat2", "incidence", "planted"])
def test_spmv_matches_oracle(ctx, oracle, which):
    import krans_b200 as kb
    from krans_b200 import generators as G
    if which == "shift":
        A = G.shift_operator(1000, 3, 0.5).A
    elif which == "mat2":
        A, _ = load_golden_matrix(2)
    elif which == "incidence":
        A = G.graph_incidence(20000, 4, 8.0, seed=3).A
    else:
        A = G.planted_kernel(3000, 2000, 8, seed=2).A
    O = oracle.Csr.from_scipy(A)
    M = kb.CudaCsrMatrixAdapter.from_scipy(ctx, A, fp32=True)
    rng = np.random.default_rng(1)
    x = rng.standard_normal(A.shape[1])
    y = rng.standard_normal(A.shape[0])
    vx, vy = kb.CudaVectorAdapter.from_numpy(ctx, x), kb.CudaVectorAdapter(ctx, A.shape[0])
    M.multiply(vx, vy)
    ref = O.matvec(x)
    scale = np.abs(A) @ np.abs(x)
    assert np.all(np.abs(vy.data() - ref) <= 1e-14 * scale + 1e-300)
    wy, wx = kb.CudaVectorAdapter.from_numpy(ctx, y), kb.CudaVectorAdapter(ctx, A.shape[1])
    M.multiply_transpose(wy, wx)
    ref = O.matvec(y, trans=True)
    scale = np.abs(A.T) @ np.abs(y)
    assert np.all(np.abs(wx.data() - ref) <= 1e-14 * scale + 1e-300)
    # FP32 values with FP32 accumulation
    M.multiply(vx, vy, precision=kb.Precision.MIXED)
    ref = A @ x
    assert np.all(np.abs(vy.data() - ref) <= 3e-6 * (np.abs(A) @ np.abs(x)) + 1e-30)
    with pytest.raises(ValueError):
        M.multiply(wy, vy)


def test_transpose_is_exact_and_deterministic(ctx):
    import ctypes as C
    import krans_b200 as kb
    from krans_b200 import generators as G
    A = G.graph_incidence(5000, 3, 7.0, seed=9).A
    outs = []
    for _ in range(2):
        M = kb.CudaCsrMatrixAdapter.from_scipy(ctx, A)
        x = kb.CudaVectorAdapter.from_numpy(ctx, np.random.default_rng(5).standard_normal(A.shape[0]))
        y = kb.CudaVectorAdapter(ctx, A.shape[1])
        M.multiply_transpose(x, y)
        outs.append(y.data())
    np.testing.assert_array_equal(outs[0], outs[1])
    np.testing.assert_allclose(outs[0], A.T @ x.data(), rtol=0, atol=1e-12)


def test_mt19937_stream_matches_libstdcxx(ctx):
    """Device MT19937 + polar normals reproduce libstdc++'s sequence: the
    uniform draws and accept/reject decisions exactly, each variate within a
    few ulp (log() may round differently from glibc's)."""
    import krans_b200 as kb
    lines = open(os.path.join(GOLDEN, "rng_normals.txt")).read().split("\n")
    i, exact, total = 0, 0, 0
    f = None
    while i < len(lines):
        t = lines[i]
        if t.startswith("seed"):
            f = kb.CudaVectorFactory(ctx, 1, seed=int(t.split()[1]))
            i += 1
        elif t.startswith("vec"):
            L = int(t.split()[1])
            want = np.array([float.fromhex(x) for x in lines[i + 1:i + 1 + L]])
            got = f.create_random_of_size(L).data()
            ulp = np.spacing(np.abs(want))
            assert np.all(np.abs(got - want) <= 4 * ulp)
            exact += int(np.sum(got == want))
            total += L
            i += 1 + L
        else:
            i += 1
    assert total == 6018 and exact >= 0.9 * total


def test_philox_stream(ctx):
    import krans_b200 as kb
    f = kb.CudaVectorFactory(ctx, 100000, seed=7, mode="philox")
    a = f.create_random().data()
    b = f.create_random().data()
    assert abs(a.mean()) < 0.02 and abs(a.std() - 1) < 0.02
    assert not np.array_equal(a, b)
    g = kb.CudaVectorFactory(ctx, 100000, seed=7, mode="philox")
    np.testing.assert_array_equal(g.create_random().data(), a)


def test_bounded_grid_barrier_wait_runs_out(ctx):
    """Failure detection without a GPU fault: a grid barrier that one block
    never reaches gives up after its bound with KRANS_ERR_TIMEOUT, and the
    context keeps working (a solve right after succeeds)."""
    import ctypes as C
    import krans_b200 as kb
    from krans_b200 import _capi as K
    from krans_b200 import generators as G
    st, ms = C.c_int(0), C.c_double(0.0)
    K.check(ctx.lib.krans_selftest_barrier_timeout(ctx.h, 300.0, C.byref(st), C.byref(ms)))
    assert st.value == K.KRANS_ERR_TIMEOUT
    assert 300.0 <= ms.value < 3000.0
    inst = G.shift_operator(1000, 3, 0.5)
    M = kb.CudaCsrMatrixAdapter.from_scipy(ctx, inst.A)
    R = kb.find_nullspace_cyclic_lanczos_ex(M, kb.CudaVectorFactory(ctx, 1000, seed=42),
                                            kb.CyclicLanczosOptions(k=3))
    assert R.converged_to_target and len(R.right_null) == 3
