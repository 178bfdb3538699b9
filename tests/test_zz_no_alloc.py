"""The allocation-free dot product (krans_vec_dot_noalloc), for callers that
cannot call cudaMalloc: it must give the same value as the allocating
krans_vec_dot, within the dot-product tolerance of the other vector tests, on
two calls in a row (the second call reuses the file-scope scratch array that
the first call left filled), called through the C ABI. This file is named so
that pytest collects it last."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_dot_noalloc_matches_allocating_dot():
    import torch
    import krans_b200 as kb
    from krans_b200 import _capi as K
    ctx = kb.Context(0)
    lib = K.load()
    rng = np.random.default_rng(11)
    for n in [0, 1, 3000, 1_000_003, 5_000_000]:
        a, b = rng.standard_normal(n), rng.standard_normal(n)
        va = kb.CudaVectorAdapter.from_numpy(ctx, a)
        vb = kb.CudaVectorAdapter.from_numpy(ctx, b)
        out = kb.CudaVectorAdapter(ctx, 1)  # the caller owns the output
        want = va.dot(vb)  # allocating entry point (context scratch)
        tol = 1e-12 * (1 + np.abs(a) @ np.abs(b))
        for _ in range(2):
            rc = lib.krans_vec_dot_noalloc(C.c_void_p(va.device_ptr()), C.c_void_p(vb.device_ptr()), n,
                                           C.c_void_p(out.device_ptr()), None)
            assert rc == 0, lib.krans_last_error()
            torch.cuda.synchronize()
            got = out.data()[0]
            assert abs(got - want) <= tol
            assert abs(got - a @ b) <= tol


def test_dot_noalloc_rejects_oversize():
    import krans_b200 as kb
    from krans_b200 import _capi as K
    kb.Context(0)
    lib = K.load()
    x = C.c_void_p(16)  # never dereferenced: the size check comes first
    rc = lib.krans_vec_dot_noalloc(x, x, (2048 * 16384) + 1, x, None)
    assert rc == K.KRANS_ERR_INVALID_ARGUMENT
    assert b"exceeds the maximum" in lib.krans_last_error()
