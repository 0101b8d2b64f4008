"""The FP16-part tensor-core GEMM on CTA pairs (context option gemm_pairs = 1:
tcgen05.mma.cta_group::2, 256-row tiles, each CTA of the pair loading half of
the tile's B operand): the same products as the one-CTA kernel -- FP32-class
error against an FP64 reference for row- and column-major operands, rows and
columns spread over 1e+-12, the lower-triangle update of the L D L^T
factorisation and its solves reaching the FP64 solution after refinement,
with first corrections of the one-CTA kernel's size."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import bem_b200 as bb
    c = bb.Context(0)
    bb.set_option(c, "tensor_split", 1)
    bb.set_option(c, "gemm_pairs", 1)
    yield c
    bb.set_option(c, "gemm_pairs", 0)
    c.close()


def _rand(shape, seed, spread=0.0):
    import torch
    g = torch.Generator().manual_seed(seed)
    z = torch.complex(torch.randn(shape, generator=g, dtype=torch.float64),
                      torch.randn(shape, generator=g, dtype=torch.float64))
    if spread:
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


@pytest.mark.parametrize("M,N,K", [(256, 128, 64), (300, 70, 100), (1000, 517, 256), (129, 300, 1), (77, 1, 33),
                                   (2048, 1024, 512)])
@pytest.mark.parametrize("b_rowmajor,c_colmajor", [(True, False), (False, True)])
def test_pair_gemm_matches_fp64(ctx, M, N, K, b_rowmajor, c_colmajor):
    import torch
    A, Bm, C0 = _rand((M, K), 1), _rand((K, N), 2), _rand((M, N), 3)
    out = _gemm(ctx, A, Bm, C0, b_rowmajor, c_colmajor)
    c64 = lambda x: x.to(torch.complex64).to(torch.complex128)
    ref32 = c64(C0) - c64(A) @ c64(Bm)
    scale = float(K) ** 0.5 * 2.0
    err = (out - ref32).abs().max().item() / scale
    assert err <= 1.5e-7 * K + 2e-6, err
    assert (out - (C0 - A @ Bm)).abs().max().item() / scale < 3e-5


def test_pair_gemm_scales_rows_and_columns(ctx):
    import torch
    M, N, K = 520, 300, 200
    A, Bm = _rand((M, K), 4, spread=6.0), _rand((K, N), 5, spread=6.0)
    out = _gemm(ctx, A, Bm, torch.zeros((M, N), dtype=torch.complex128), True, False)
    ref = -(A.to(torch.complex64).to(torch.complex128) @ Bm.to(torch.complex64).to(torch.complex128))
    assert torch.isfinite(out).all()
    assert ((out - ref).abs() / (A.abs() @ Bm.abs())).max().item() < 2e-5


def test_pair_ldlt_on_pmchwt_matches_one_cta_kernel(ctx):
    # L D L^T of the assembled PMCHWT system (2N = 3840: lower-triangle
    # updates with K = 512, the panel in store mode, the solves' updates)
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
    try:
        for pairs in (1, 0):
            bb.set_option(ctx, "gemm_pairs", pairs)
            lu = bb.LU(ctx, Z, bb.PREC_FP32_REFINE)
            X, st = lu.solve(B, tol=2e-10, max_iter=12)
            lu.close()
            res[pairs] = (X.cpu().numpy(), st)
    finally:
        bb.set_option(ctx, "gemm_pairs", 1)
    X64h = X64.cpu().numpy()
    for pairs, (X, st) in res.items():
        assert st["converged"] == 1 and st["factorization"] == 2, (pairs, st)
        col = np.linalg.norm(X - X64h, axis=1) / np.linalg.norm(X64h, axis=1)
        assert col.max() < 1e-9, (pairs, col.max())
    u1, u0 = res[1][1]["update_hist"][0], res[0][1]["update_hist"][0]
    assert u1 < 2 * u0 and u0 < 2 * u1, (u1, u0)
    g.close()
