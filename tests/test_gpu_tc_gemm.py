"""The 3xTF32 tcgen05 complex GEMM against an FP64 torch reference.

Tolerance: the result must be FP32-class.  Its max error against the FP64
product of the complex64-rounded inputs is compared with that of an FP32
CUDA-core GEMM (torch complex64 matmul, TF32 off) on the same inputs.  The
tensor core's FP32 accumulation inside one MMA chain does not round to
nearest; measured on B200 its error grows about linearly with the K of one
call (13x the CUDA-core error at K = 256 complex), so the bound is
max(4 err_fp32, 1.5e-7 K) in units of 2 sqrt(K) (an entry's magnitude)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    # the TF32 split (tensor_split 0); the FP16 split has its own tests
    import bem_b200 as bb
    c = bb.Context(0)
    bb.set_option(c, "tensor_split", 0)
    yield c
    c.close()


def _rand(shape, seed):
    import torch
    g = torch.Generator().manual_seed(seed)
    re = torch.randn(shape, generator=g, dtype=torch.float64)
    im = torch.randn(shape, generator=g, dtype=torch.float64)
    return torch.complex(re, im)


@pytest.mark.parametrize("M,N,K", [(128, 128, 16), (300, 70, 100), (1000, 517, 256),
                                   (129, 129, 1), (77, 1, 33)])
@pytest.mark.parametrize("b_rowmajor,c_colmajor", [(True, False), (False, True)])
def test_tc_gemm_matches_fp64(ctx, M, N, K, b_rowmajor, c_colmajor):
    import torch
    import bem_b200 as bb
    A = _rand((M, K), 1)
    Bm = _rand((K, N), 2)
    C0 = _rand((M, N), 3)
    ref = C0 - A @ Bm
    Ad = A.to(torch.complex64).cuda()
    Bd = (Bm if b_rowmajor else Bm.T.contiguous()).to(torch.complex64).cuda()
    Cd = (C0 if not c_colmajor else C0.T.contiguous()).to(torch.complex64).cuda()
    bb.cgemm_tf32x3(ctx, Ad, Bd, Cd, b_rowmajor=b_rowmajor, c_colmajor=c_colmajor)
    out = Cd.cpu().to(torch.complex128)
    if c_colmajor:
        out = out.T
    # inputs are rounded to complex64 first; compare against that rounding too
    ref32 = C0.to(torch.complex64).to(torch.complex128) - (A.to(torch.complex64).to(torch.complex128)
                                                           @ Bm.to(torch.complex64).to(torch.complex128))
    scale = float(K) ** 0.5 * 2.0
    err = (out - ref32).abs().max().item() / scale
    torch.backends.cuda.matmul.allow_tf32 = False
    f32 = (C0.to(torch.complex64).cuda() - A.to(torch.complex64).cuda() @ Bm.to(torch.complex64).cuda())
    err32 = (f32.cpu().to(torch.complex128) - ref32).abs().max().item() / scale
    assert err <= max(4 * err32, 1.5e-7 * K) + 1e-6, (err, err32)
    assert (out - ref).abs().max().item() / scale < 3e-5


def test_fp32_lu_on_tensor_cores_matches_cuda_cores(ctx):
    # same FP32 factorisation with the tensor-core and CUDA-core updates
    import torch
    import bem_b200 as bb
    n = 700
    A = _rand((n, n), 9) + 3 * n ** 0.5 * torch.eye(n, dtype=torch.complex128)
    B = _rand((5, n), 10)
    res = {}
    for tc in (True, False):
        bb.set_tensor_cores(ctx, tc)
        lu = bb.LU(ctx, A.cuda().contiguous(), bb.PREC_FP32_REFINE)
        X, st = lu.solve(B.cuda(), tol=1e-13)
        res[tc] = (X.cpu(), st)
    bb.set_tensor_cores(ctx, True)
    Xr = torch.linalg.solve(A, B.T).T
    for tc, (X, st) in res.items():
        assert st["converged"] == 1
        assert ((X - Xr).abs().max() / Xr.abs().max()).item() < 1e-11, (tc, st)
