"""Int8 tensor-core (Ozaki scheme) FP64 refinement residual R = B - Z X.

Both residual methods are checked against an extended-precision (x87 80-bit,
64-bit significand) evaluation of the same product on the host.  With S
digits every entry is kept to 2^(1-7S) of its row (column) maximum and the
dropped digit pairs weigh about as much again, so a product term is good to
about 2^(3-7S) max|Z| max|X|; the bound used here is 2^(4-7S) sqrt(2n)
max|Z| max|X| (a random walk over the 2n real terms).  8 digits must match
the FP64 GEMM within a small factor.
Rows and columns whose scales differ by hundreds of binades are covered by
the per-row / per-column exponents."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bound(n, digits=7):
    return 2.0 ** (4 - 7 * digits) * np.sqrt(2.0 * n)


@pytest.fixture(scope="module")
def ctx():
    import bem_b200 as bb
    c = bb.Context(0)
    yield c
    c.close()


def _cplx(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def _exact_residual(Z, X, B):
    """B - Z X in clongdouble (columns of X / B are rows of the arrays)."""
    Zl = Z.astype(np.clongdouble)
    Xl = X.astype(np.clongdouble)
    return B.astype(np.clongdouble) - Xl @ Zl.T


def _run(ctx, Z, X, B, digits=7):
    import torch
    import bem_b200 as bb
    bb.set_residual_digits(ctx, digits)
    try:
        Zt = torch.from_numpy(Z.copy()).cuda()
        lu = bb.LU(ctx, Zt, bb.PREC_FP32_REFINE)
        Bt = torch.from_numpy(B.copy()).cuda()
        Xt = torch.from_numpy(X.copy()).cuda()
        R64 = lu.residual(Bt, Xt, method=0).cpu().numpy()
        Roz = lu.residual(Bt, Xt, method=1).cpu().numpy() if digits else None
        lu.close()
    finally:
        bb.set_residual_digits(ctx, 7)
    return R64, Roz


@pytest.mark.parametrize("n,nrhs", [(1, 1), (37, 3), (128, 128), (300, 129), (1000, 70)])
def test_ozaki_matches_fp64(ctx, n, nrhs):
    rng = np.random.default_rng(1000 + n)
    Z = _cplx(rng, n, n)
    X = _cplx(rng, nrhs, n)
    B = _cplx(rng, nrhs, n)
    Re = _exact_residual(Z, X, B)
    scale = np.abs(Z).max() * np.abs(X).max()
    R64, Roz = _run(ctx, Z, X, B, digits=7)
    e64 = float(np.abs(R64 - Re).max()) / scale
    eoz = float(np.abs(Roz - Re).max()) / scale
    assert eoz < _bound(n), (eoz, e64)
    _, Roz8 = _run(ctx, Z, X, B, digits=8)
    eoz8 = float(np.abs(Roz8 - Re).max()) / scale
    assert eoz8 < 4 * max(e64, 1e-16 * np.sqrt(n)), (eoz8, e64)


def test_ozaki_small_residual_cancellation(ctx):
    # refinement regime: B ~ Z X, R is 1e-8 of B; the error must be absolute
    # FP64-level, not relative to R
    n, nrhs = 512, 40
    rng = np.random.default_rng(7)
    Z = _cplx(rng, n, n)
    X = _cplx(rng, nrhs, n)
    B = (X.astype(np.clongdouble) @ Z.astype(np.clongdouble).T).astype(np.complex128)
    B += 1e-8 * _cplx(rng, nrhs, n)
    R64, Roz = _run(ctx, Z, X, B)
    Re = _exact_residual(Z, X, B)
    scale = np.abs(Z).max() * np.abs(X).max()
    e64 = float(np.abs(R64 - Re).max()) / scale
    eoz = float(np.abs(Roz - Re).max()) / scale
    assert eoz < _bound(n), (eoz, e64)


def test_ozaki_extreme_row_and_column_scales(ctx):
    n, nrhs = 300, 20
    rng = np.random.default_rng(11)
    Z = _cplx(rng, n, n) + 20.0 * np.eye(n)   # keeps the FP32 factorisation away from overflow
    X = _cplx(rng, nrhs, n)
    X[3] *= 2.0 ** 400
    X[5] *= 2.0 ** -500
    X[7] = 0.0                                  # zero column: exponent 0, digits 0
    Z[:, 17] *= 1e-3
    B = _cplx(rng, nrhs, n)
    B[3] *= 2.0 ** 400
    B[5] *= 2.0 ** -500
    R64, Roz = _run(ctx, Z, X, B)
    Re = _exact_residual(Z, X, B)
    for j in range(nrhs):
        scale = np.abs(Z).max() * max(np.abs(X[j]).max(), np.abs(B[j]).max() / n)
        e = float(np.abs(Roz[j] - Re[j]).max()) / scale
        assert e < _bound(n), (j, e)
    assert np.array_equal(Roz[7], B[7])


def test_fewer_digits_degrade_gracefully(ctx):
    n, nrhs = 256, 16
    rng = np.random.default_rng(3)
    Z = _cplx(rng, n, n)
    X = _cplx(rng, nrhs, n)
    B = _cplx(rng, nrhs, n)
    Re = _exact_residual(Z, X, B)
    scale = np.abs(Z).max() * np.abs(X).max()
    errs = []
    for d in (3, 5, 7):
        _, Roz = _run(ctx, Z, X, B, digits=d)
        errs.append(float(np.abs(Roz - Re).max()) / scale)
    # each two extra digits buy ~14 bits
    assert errs[0] > 100 * errs[1] > 100 * 100 * errs[2] / 10, errs
    assert errs[0] < n * 2.0 ** (-7 * 3 + 2)


def test_refinement_with_and_without_ozaki_agree(ctx):
    import torch
    import bem_b200 as bb
    n, nrhs = 700, 30
    rng = np.random.default_rng(5)
    A = _cplx(rng, n, n)
    B = _cplx(rng, n, nrhs)
    out = []
    for d in (0, 7):
        bb.set_residual_digits(ctx, d)
        Zt = torch.from_numpy(A.copy()).cuda()
        lu = bb.LU(ctx, Zt, bb.PREC_FP32_REFINE)
        X, st = lu.solve(B, tol=1e-12)
        assert st["converged"]
        out.append(X.cpu().numpy().T)
        lu.close()
    bb.set_residual_digits(ctx, 7)
    Xr = np.linalg.solve(A, B)
    for X in out:
        assert np.abs(X - Xr).max() / np.abs(Xr).max() < 1e-10


def test_residual_method_needs_digit_planes(ctx):
    import torch
    import bem_b200 as bb
    bb.set_residual_digits(ctx, 0)
    try:
        Zt = torch.eye(64, dtype=torch.complex128, device="cuda")
        lu = bb.LU(ctx, Zt, bb.PREC_FP32_REFINE)
        B = torch.ones(2, 64, dtype=torch.complex128, device="cuda")
        with pytest.raises(bb.BemError):
            lu.residual(B, B, method=1)
        R = lu.residual(B, B, method=0)
        assert float(R.abs().max()) == 0.0
        lu.close()
    finally:
        bb.set_residual_digits(ctx, 7)
    with pytest.raises(bb.BemError):
        bb.set_residual_digits(ctx, 9)


@pytest.mark.parametrize("n,nrhs", [(1, 1), (300, 129), (700, 300)])
def test_pacing_does_not_change_the_residual(ctx, n, nrhs):
    # the producers' pacing (residual_pace_epoch / residual_pace_lead) only
    # delays TMA loads: every tile still sums the same integer products in
    # the same group order, so the residual is bitwise the same
    import torch
    import bem_b200 as bb
    rng = np.random.default_rng(77 + n)
    Z = _cplx(rng, n, n) + 3 * np.eye(n)
    X = _cplx(rng, nrhs, n)
    B = _cplx(rng, nrhs, n)
    Zt = torch.from_numpy(Z.copy()).cuda()
    lu = bb.LU(ctx, Zt, bb.PREC_FP32_REFINE)
    Bt = torch.from_numpy(B.copy()).cuda()
    Xt = torch.from_numpy(X.copy()).cuda()
    out = []
    try:
        for epoch, lead in ((32, 2), (0, 2), (1, 0)):
            bb.set_option(ctx, "residual_pace_epoch", epoch)
            bb.set_option(ctx, "residual_pace_lead", lead)
            out.append(lu.residual(Bt, Xt, method=1).cpu().numpy())
    finally:
        bb.set_option(ctx, "residual_pace_epoch", 32)
        bb.set_option(ctx, "residual_pace_lead", 2)
        lu.close()
    assert all(np.array_equal(out[0], R) for R in out[1:])
    with pytest.raises(bb.BemError):
        bb.set_option(ctx, "no_such_option", 1)
