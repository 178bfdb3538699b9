"""The block solver's dense products on their own (krans_block_gram,
krans_block_gemm_tn, krans_block_combine: the device code LOBPCG runs inside
its kernel) against numpy: S = Z^T Z and G = Z^T W formed on the upper
triangle and mirrored, as the reference's form_gram does
(LOBPCGSolver.cpp:67-80), C = A^T B as the basis projections of
orthonormalize_block (LOBPCGSolver.cpp:137-160), and out = Z C as
combine_columns (LOBPCGSolver.cpp:122-134). Tolerance: 64 ulp of the sum of
absolute products of each entry."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
EPS = 2.220446049250313e-16


def dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).to("cuda:0")


@pytest.mark.parametrize("n,p", [(1, 1), (1000, 3), (200_001, 40), (131_073, 96), (300_000, 200)])
def test_block_gram(ctx, n, p):
    import torch
    import krans_b200 as kb
    rng = np.random.default_rng(n + p)
    ld = n + (7 if n > 1 else 0)
    Zc = rng.standard_normal((p, ld))  # column j of the n x p block = row j (leading dimension ld)
    Wc = rng.standard_normal((p, ld))
    Z, W = dev(Zc), dev(Wc)
    S, G = torch.zeros(p, p, dtype=torch.float64, device="cuda:0"), torch.zeros(p, p, dtype=torch.float64,
                                                                                   device="cuda:0")
    torch.cuda.synchronize()
    kb.block_gram(ctx, n, p, Z.data_ptr(), ld, S.data_ptr(), W.data_ptr(), G.data_ptr())
    Zn, Wn = Zc[:, :n].T, Wc[:, :n].T
    Sref, Gu = Zn.T @ Zn, Zn.T @ Wn
    Gref = np.triu(Gu) + np.triu(Gu, 1).T  # upper triangle mirrored
    tol_s = 64 * EPS * (np.abs(Zn).T @ np.abs(Zn))
    tol_g = 64 * EPS * (np.abs(Zn).T @ np.abs(Wn))
    tol_g = np.triu(tol_g) + np.triu(tol_g, 1).T
    Sd, Gd = S.cpu().numpy().T, G.cpu().numpy().T  # column-major p x p
    assert np.all(np.abs(Sd - Sref) <= tol_s) and np.array_equal(Sd, Sd.T)
    assert np.all(np.abs(Gd - Gref) <= tol_g) and np.array_equal(Gd, Gd.T)
    S2 = torch.zeros_like(S)
    kb.block_gram(ctx, n, p, Z.data_ptr(), ld, S2.data_ptr())  # S alone
    assert torch.equal(S2, S)


@pytest.mark.parametrize("n,a,b", [(1, 1, 1), (1000, 5, 3), (131_072, 64, 96), (300_001, 40, 7),
                                   (200_000, 130, 70)])
def test_block_gemm_tn(ctx, n, a, b):
    # n >= 131072 with a or b >= 32: the shared-memory panel form; else one
    # warp per 8 x 8 output tile
    import torch
    import krans_b200 as kb
    rng = np.random.default_rng(n + a + b)
    ld = n + 5
    Ac, Bc = rng.standard_normal((a, ld)), rng.standard_normal((b, ld))
    A, B = dev(Ac), dev(Bc)
    Cd = torch.full((b, a), 3.0, dtype=torch.float64, device="cuda:0")
    torch.cuda.synchronize()
    kb.block_gemm_tn(ctx, n, a, A.data_ptr(), b, B.data_ptr(), ld, Cd.data_ptr())
    An, Bn = Ac[:, :n].T, Bc[:, :n].T
    ref = An.T @ Bn
    tol = 64 * EPS * (np.abs(An).T @ np.abs(Bn))
    got = Cd.cpu().numpy().T  # column-major a x b
    assert np.all(np.abs(got - ref) <= tol)
    C2 = torch.zeros_like(Cd)
    kb.block_gemm_tn(ctx, n, a, A.data_ptr(), b, B.data_ptr(), ld, C2.data_ptr())
    assert torch.equal(C2, Cd)  # deterministic


@pytest.mark.parametrize("n,zc,q", [(1, 1, 1), (1000, 3, 3), (200_001, 96, 96), (70_000, 288, 96), (5000, 40, 300)])
def test_block_combine(ctx, n, zc, q):
    import torch
    import krans_b200 as kb
    rng = np.random.default_rng(n + zc + q)
    ld = n + 3
    Zc = rng.standard_normal((zc, ld))
    Cm = rng.standard_normal((q, zc + 2))  # column-major zc x q with leading dimension zc + 2
    Z, Cd = dev(Zc), dev(Cm)
    out = torch.full((q, ld), 7.0, dtype=torch.float64, device="cuda:0")
    torch.cuda.synchronize()
    kb.block_combine(ctx, n, zc, q, Z.data_ptr(), ld, Cd.data_ptr(), zc + 2, out.data_ptr())
    Zn, Cn = Zc[:, :n].T, Cm[:, :zc].T
    ref = Zn @ Cn
    tol = 64 * EPS * (np.abs(Zn) @ np.abs(Cn))
    got = out.cpu().numpy()
    assert np.all(np.abs(got[:, :n].T - ref) <= tol)
    assert np.all(got[:, n:] == 7.0)  # padding rows untouched


def test_block_products_invalid(ctx):
    import krans_b200 as kb
    with pytest.raises(ValueError):
        kb.block_gram(ctx, 10, 0, 16, 10, 16)
    with pytest.raises(ValueError):
        kb.block_gram(ctx, 10, 3, 16, 5, 16)  # ld < n
    with pytest.raises(ValueError):
        kb.block_gram(ctx, 10, 3, 16, 10, 16, W=16)  # W without G
    with pytest.raises(ValueError):
        kb.block_combine(ctx, 10, 3, 2, 16, 10, 16, 2, 16)  # ldc < zc
    with pytest.raises(ValueError):
        kb.block_gemm_tn(ctx, 10, 3, 16, 2, 16, 9, 16)  # ld < n
