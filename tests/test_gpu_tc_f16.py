"""The tensor-core GEMM with FP16 operand parts (context option
tensor_split = 1): every row of A' and complex column of B is scaled by a
power of two into [2^14, 2^15) and split into two FP16 parts, the products
hi*hi + hi*lo + lo*hi are taken with tcgen05 kind::f16 and the epilogue
undoes the scales.  FP16 carries the same 11 significant bits as TF32, so the
bar is the 3xTF32 path's: FP32-class error against an FP64 reference, the
FP32 factorisations reaching FP64 accuracy after refinement, and results
close to the TF32 split's."""
import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import bem_b200 as bb
    c = bb.Context(0)
    bb.set_option(c, "tensor_split", 1)
    yield c
    bb.set_option(c, "tensor_split", 0)
    c.close()


def _rand(shape, seed, spread=0.0):
    import torch
    g = torch.Generator().manual_seed(seed)
    re = torch.randn(shape, generator=g, dtype=torch.float64)
    im = torch.randn(shape, generator=g, dtype=torch.float64)
    z = torch.complex(re, im)
    if spread:
        # rows and columns of very different magnitudes (1e-spread .. 1e+spread)
        r = 10.0 ** (spread * (2 * torch.rand(shape[0], generator=g, dtype=torch.float64) - 1))
        c = 10.0 ** (spread * (2 * torch.rand(shape[1], generator=g, dtype=torch.float64) - 1))
        z = z * r[:, None] * c[None, :]
    return z


def _gemm(ctx, A, Bm, C0, b_rowmajor, c_colmajor):
    import torch
    import bem_b200 as bb
    Ad = A.to(torch.complex64).cuda()
    Bd = (Bm if b_rowmajor else Bm.T.contiguous()).to(torch.complex64).cuda()
    Cd = (C0 if not c_colmajor else C0.T.contiguous()).to(torch.complex64).cuda()
    bb.cgemm_tf32x3(ctx, Ad, Bd, Cd, b_rowmajor=b_rowmajor, c_colmajor=c_colmajor)
    out = Cd.cpu().to(torch.complex128)
    return out.T if c_colmajor else out


@pytest.mark.parametrize("M,N,K", [(128, 128, 16), (300, 70, 100), (1000, 517, 256), (129, 129, 1), (77, 1, 33)])
@pytest.mark.parametrize("b_rowmajor,c_colmajor", [(True, False), (False, True)])
def test_f16_split_gemm_matches_fp64(ctx, M, N, K, b_rowmajor, c_colmajor):
    import torch
    A, Bm, C0 = _rand((M, K), 1), _rand((K, N), 2), _rand((M, N), 3)
    out = _gemm(ctx, A, Bm, C0, b_rowmajor, c_colmajor)
    c64 = lambda x: x.to(torch.complex64).to(torch.complex128)
    ref32 = c64(C0) - c64(A) @ c64(Bm)
    scale = float(K) ** 0.5 * 2.0
    err = (out - ref32).abs().max().item() / scale
    # the 3xTF32 bound of the same test (FP32-class, MMA-chain accumulation)
    assert err <= 1.5e-7 * K + 1e-6, err
    assert (out - (C0 - A @ Bm)).abs().max().item() / scale < 3e-5


def test_f16_split_scales_rows_and_columns(ctx):
    # entries spanning 1e-12 .. 1e+12 across rows and columns: without the
    # per-row / per-column scales FP16 would overflow and underflow
    import torch
    M, N, K = 260, 300, 200
    A, Bm = _rand((M, K), 4, spread=6.0), _rand((K, N), 5, spread=6.0)
    C0 = torch.zeros((M, N), dtype=torch.complex128)
    out = _gemm(ctx, A, Bm, C0, True, False)
    ref = -(A.to(torch.complex64).to(torch.complex128) @ Bm.to(torch.complex64).to(torch.complex128))
    # entrywise against |A| |B|, the scale of each product sum (FP32
    # accumulation: about 2e-7 sqrt(K) of it; a wrong scale gives O(1) or inf)
    bound = (A.abs() @ Bm.abs())
    assert torch.isfinite(out).all()
    assert ((out - ref).abs() / bound).max().item() < 2e-5


def test_f16_split_lu_and_ldlt_reach_fp64(ctx):
    import torch
    import bem_b200 as bb
    n = 700
    A = _rand((n, n), 9) + 3 * n ** 0.5 * torch.eye(n, dtype=torch.complex128)
    B = _rand((5, n), 10)
    Xr = torch.linalg.solve(A, B.T).T
    lu = bb.LU(ctx, A.cuda().contiguous(), bb.PREC_FP32_REFINE)
    X, st = lu.solve(B.cuda(), tol=1e-13)
    lu.close()
    assert st["converged"] == 1
    assert ((X.cpu() - Xr).abs().max() / Xr.abs().max()).item() < 1e-11, st


def test_f16_split_pmchwt_ldlt_matches_tf32_split(ctx):
    # the assembled PMCHWT system through the symmetric L D L^T path, with
    # K = 512 super-block updates and the solves' transposed-A packing
    import torch
    import bem_b200 as bb
    v, t = bb.icosphere(1.0, 3)
    kx, ki, ee, ei = bb.physics(5.0, complex(1.3116, 1e-4))
    g = bb.Geometry(ctx, v, t, 7)
    Z = bb.assemble_pmchwt_dev(g, kx, ki, ee, ei)
    RT, w = bb.generate_orientations(4, 3, 1)
    B = bb.rhs_planewave_dev(g, kx, ee, RT)
    lu64 = bb.LU(ctx, Z.clone(), bb.PREC_FP64)
    X64, _ = lu64.solve(B)
    lu64.close()
    res = {}
    for split in (1, 0):
        bb.set_option(ctx, "tensor_split", split)
        lu = bb.LU(ctx, Z, bb.PREC_FP32_REFINE)
        X, st = lu.solve(B, tol=2e-10, max_iter=12)
        lu.close()
        res[split] = (X.cpu().numpy(), st)
    bb.set_option(ctx, "tensor_split", 1)
    X64h = X64.cpu().numpy()
    for split, (X, st) in res.items():
        assert st["converged"] == 1 and st["factorization"] == 2, (split, st)
        col = np.linalg.norm(X - X64h, axis=1) / np.linalg.norm(X64h, axis=1)
        assert col.max() < 1e-9, (split, col.max())
    # the first correction (the FP32 solve's own error) is of the same size
    u1, u0 = res[1][1]["update_hist"][0], res[0][1]["update_hist"][0]
    assert u1 < 4 * u0 and u0 < 4 * u1, (u1, u0)
    g.close()
