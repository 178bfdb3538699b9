"""The allocation-free dot product (krans_vec_dot_noalloc), for callers that
cannot call cudaMalloc: it must give the same value as the allocating
krans_vec_dot, within the dot-product tolerance of the other vector tests, on
two calls in a row (the second call reuses the file-scope scratch array that
the first call left filled), called through the C ABI, on the legacy default
stream and on a caller's own stream. After the first call (which looks up the
array's address and loads the kernels) further calls must leave the device's
free memory and torch's allocator untouched. This file is named so that
pytest collects it last."""
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
    side = torch.cuda.Stream(device=0)
    for n in [0, 1, 3000, 1_000_003, 5_000_000]:
        a, b = rng.standard_normal(n), rng.standard_normal(n)
        va = kb.CudaVectorAdapter.from_numpy(ctx, a)
        vb = kb.CudaVectorAdapter.from_numpy(ctx, b)
        out = kb.CudaVectorAdapter(ctx, 1)  # the caller owns the output
        want = va.dot(vb)  # allocating entry point (context scratch); synchronizes the context
        tol = 1e-12 * (1 + np.abs(a) @ np.abs(b))
        for stream in (None, C.c_void_p(side.cuda_stream)):
            for _ in range(2):
                rc = lib.krans_vec_dot_noalloc(C.c_void_p(va.device_ptr()), C.c_void_p(vb.device_ptr()), n,
                                               C.c_void_p(out.device_ptr()), stream)
                assert rc == 0, lib.krans_last_error()
                if stream is None:
                    torch.cuda.synchronize()
                else:
                    side.synchronize()
                got = out.data()[0]
                assert abs(got - want) <= tol
                assert abs(got - a @ b) <= tol


def test_dot_noalloc_allocates_nothing():
    import torch
    import krans_b200 as kb
    from krans_b200 import _capi as K
    ctx = kb.Context(0)
    lib = K.load()
    n = 4_000_000
    rng = np.random.default_rng(12)
    a, b = rng.standard_normal(n), rng.standard_normal(n)
    va, vb = kb.CudaVectorAdapter.from_numpy(ctx, a), kb.CudaVectorAdapter.from_numpy(ctx, b)
    out = kb.CudaVectorAdapter(ctx, 1)
    side = torch.cuda.Stream(device=0)
    args = (C.c_void_p(va.device_ptr()), C.c_void_p(vb.device_ptr()), n, C.c_void_p(out.device_ptr()))
    assert lib.krans_vec_dot_noalloc(*args, None) == 0  # first call: address lookup, kernel loading
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    torch0 = torch.cuda.memory_allocated(0)
    for stream in (None, C.c_void_p(side.cuda_stream)) * 4:
        assert lib.krans_vec_dot_noalloc(*args, stream) == 0, lib.krans_last_error()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0
    assert torch.cuda.memory_allocated(0) == torch0
    assert abs(out.data()[0] - a @ b) <= 1e-12 * (1 + np.abs(a) @ np.abs(b))


def test_dot_noalloc_rejects_oversize():
    import krans_b200 as kb
    from krans_b200 import _capi as K
    kb.Context(0)
    lib = K.load()
    x = C.c_void_p(16)  # never dereferenced: the size check comes first
    rc = lib.krans_vec_dot_noalloc(x, x, (2048 * 16384) + 1, x, None)
    assert rc == K.KRANS_ERR_INVALID_ARGUMENT
    assert b"exceeds the maximum" in lib.krans_last_error()
