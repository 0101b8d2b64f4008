"""FP32 L D L^T without pivoting for symmetric-structured systems.

The PMCHWT Z is [[A, -K], [K, C]] with A, C, K symmetric, so Z diag(I, -I)
is symmetric; the FP32 + refinement solve factors it as L D L^T (half the
flops of LU) and must give the FP64 solution.  Plain symmetric matrices use
the same path with s = 1; a zero pivot, or a factorisation too inaccurate for
the refinement to converge, falls back to LU with partial pivoting."""
import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import bem_b200 as bb
    c = bb.Context(0)
    yield c
    bb.set_symmetric(c, 1)
    c.close()


def _solve(ctx, Z, B, sym=1, tol=1e-12):
    import torch
    import bem_b200 as bb
    bb.set_symmetric(ctx, sym)
    try:
        Zt = torch.from_numpy(np.ascontiguousarray(Z)).cuda()
        lu = bb.LU(ctx, Zt, bb.PREC_FP32_REFINE)
        X, st = lu.solve(B, tol=tol, max_iter=12)
        lu.close()
    finally:
        bb.set_symmetric(ctx, 1)
    return X.cpu().numpy().T, st


def _cplx(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


@pytest.fixture(scope="module")
def pmchwt():
    import bem_b200 as bb
    c = bb.Context(0)
    v, t = bb.icosphere(1.0, 3)
    kx, ki, ee, ei = bb.physics(5.0, complex(1.3116, 1e-4))
    g = bb.Geometry(c, v, t, 7)
    Z = bb.assemble_pmchwt_dev(g, kx, ki, ee, ei).cpu().numpy()
    RT, w = bb.generate_orientations(4, 3, 1)
    B = bb.rhs_planewave_dev(g, kx, ee, RT).cpu().numpy().T
    g.close()
    c.close()
    return Z, B


def test_pmchwt_structure_is_symmetric_after_sign_flip(pmchwt):
    Z, _ = pmchwt
    n = Z.shape[0]
    S = Z.copy()
    S[:, n // 2:] *= -1
    assert np.array_equal(S, S.T)
    assert not np.array_equal(Z, Z.T)


def test_pmchwt_ldlt_matches_fp64(ctx, pmchwt):
    import scipy.linalg as sl
    Z, B = pmchwt
    X1, st1 = _solve(ctx, Z, B, sym=1)
    X0, st0 = _solve(ctx, Z, B, sym=0)
    assert st1["factorization"] == 2 and st0["factorization"] == 0
    assert st1["converged"] and st0["converged"]
    Xr = sl.lu_solve(sl.lu_factor(Z), B)
    for X in (X1, X0):
        err = np.linalg.norm(X - Xr, axis=0) / np.linalg.norm(Xr, axis=0)
        assert err.max() < 1e-10
    # the no-pivot factors are about as good a preconditioner as partial pivoting
    assert st1["update_hist"][0] < 20 * st0["update_hist"][0]


@pytest.mark.parametrize("case", ["pmchwt", 300, 700])
def test_block_inverse_solves_match_triangular_solves(ctx, pmchwt, case):
    # solve_block_inverse (default): the diagonal blocks of the L D L^T solves
    # as tensor-core products with the stored -L11^-1; 0: block triangular
    # solves.  Both converge to the FP64 solution and precondition alike
    # (ragged last blocks for n = 300, 700)
    import scipy.linalg as sl
    import bem_b200 as bb
    if case == "pmchwt":
        Z, B = pmchwt
        sym = 1
    else:
        rng = np.random.default_rng(case)
        A = _cplx(rng, case, case)
        Z = A + A.T + 4 * np.sqrt(case) * np.eye(case)
        B = _cplx(rng, case, 9)
        sym = 1
    Xr = sl.lu_solve(sl.lu_factor(Z), B)
    out = {}
    try:
        for inv in (1, 0):
            bb.set_option(ctx, "solve_block_inverse", inv)
            out[inv] = _solve(ctx, Z, B, sym=sym)
    finally:
        bb.set_option(ctx, "solve_block_inverse", 1)
    for X, st in out.values():
        assert st["factorization"] in (1, 2) and st["converged"]
        err = np.linalg.norm(X - Xr, axis=0) / np.linalg.norm(Xr, axis=0)
        assert err.max() < 1e-10
    u1, u0 = out[1][1]["update_hist"][0], out[0][1]["update_hist"][0]
    assert u1 < 3 * u0, (u1, u0)


@pytest.mark.parametrize("case", ["pmchwt", 100, 300, 1100])
def test_cluster_diagonal_blocks_match_one_cta(ctx, pmchwt, case):
    # ldlt_cluster_diag (default): the 256 x 256 diagonal blocks of the
    # L D L^T factored by an 8-CTA cluster holding the block in distributed
    # shared memory; 0: by one CTA.  Both take every entry through the same
    # operations in the same order, so the solutions agree to the last bits
    # of the refinement; n = 100, 300, 1100 leave ragged last blocks and
    # partial 32-column sub-panels
    import scipy.linalg as sl
    import bem_b200 as bb
    if case == "pmchwt":
        Z, B = pmchwt
    else:
        rng = np.random.default_rng(case)
        A = _cplx(rng, case, case)
        Z = A + A.T + 4 * np.sqrt(case) * np.eye(case)
        B = _cplx(rng, case, 5)
    Xr = sl.lu_solve(sl.lu_factor(Z), B)
    out = {}
    try:
        for cl in (1, 0):
            bb.set_option(ctx, "ldlt_cluster_diag", cl)
            out[cl] = _solve(ctx, Z, B)
    finally:
        bb.set_option(ctx, "ldlt_cluster_diag", 1)
    for X, st in out.values():
        assert st["factorization"] in (1, 2) and st["converged"]
        err = np.linalg.norm(X - Xr, axis=0) / np.linalg.norm(Xr, axis=0)
        assert err.max() < 1e-10
    (X1, s1), (X0, s0) = out[1], out[0]
    assert rel(X1, X0) < 1e-12
    assert s1["update_hist"][0] == pytest.approx(s0["update_hist"][0], rel=1e-3)


@pytest.mark.parametrize("fsb,ssb", [(1, 1), (2, 2), (3, 4), (4, 3)])
def test_superblocks_of_any_width_solve(ctx, fsb, ssb):
    # factor_superblock / solve_superblock 1..4: the diagonal blocks of a
    # super-block update one another, the rest is updated once with K = 256 sb;
    # n = 1100 leaves a ragged last block and a short last super-block
    import bem_b200 as bb
    rng = np.random.default_rng(fsb * 10 + ssb)
    n = 1100
    A = _cplx(rng, n, n)
    Z = A + A.T + 4 * np.sqrt(n) * np.eye(n)
    B = _cplx(rng, n, 7)
    try:
        bb.set_option(ctx, "factor_superblock", fsb)
        bb.set_option(ctx, "solve_superblock", ssb)
        X, st = _solve(ctx, Z, B)
    finally:
        bb.set_option(ctx, "factor_superblock", 4)
        bb.set_option(ctx, "solve_superblock", 4)
    assert st["factorization"] == 1 and st["converged"]
    assert rel(X, np.linalg.solve(Z, B)) < 1e-11
    with pytest.raises(bb.BemError):
        bb.set_option(ctx, "factor_superblock", 5)


@pytest.mark.parametrize("xd", [3, 2])
def test_rounded_iterates_keep_the_fp64_solution(ctx, pmchwt, xd):
    # residual_x_digits (default 2): the first iterate and the corrections are
    # rounded to their first digits and kept so; the int8 residual then needs
    # fewer digit pairs and is exact for the rounded iterate, so the refined
    # solution is the FP64 one as with every digit (0)
    import scipy.linalg as sl
    import bem_b200 as bb
    Z, B = pmchwt
    Xr = sl.lu_solve(sl.lu_factor(Z), B)
    out = {}
    try:
        for d in (xd, 0):
            bb.set_option(ctx, "residual_x_digits", d)
            out[d] = _solve(ctx, Z, B, tol=2e-10)
    finally:
        bb.set_option(ctx, "residual_x_digits", 2)
    for X, st in out.values():
        assert st["converged"]
        err = np.linalg.norm(X - Xr, axis=0) / np.linalg.norm(Xr, axis=0)
        assert err.max() < 1e-10
        assert st["verified_rel_error"] < 1e-9
    assert out[xd][1]["iterations"] <= out[0][1]["iterations"] + 1


def test_rounded_iterates_with_zero_and_extreme_columns(ctx, pmchwt):
    # the rounding is relative to each column's largest entry: a zero column
    # stays exactly zero, columns scaled by 1e-150 / 1e+150 converge like the
    # others (the digit exponents follow the column)
    import scipy.linalg as sl
    Z, B0 = pmchwt
    B = B0[:, :6].copy()
    B[:, 0] = 0.0
    B[:, 1] *= 1e-150
    B[:, 2] *= 1e150
    X, st = _solve(ctx, Z, B, tol=2e-10)
    assert st["converged"]
    assert np.all(X[:, 0] == 0)
    Xr = sl.lu_solve(sl.lu_factor(Z), B)
    err = np.linalg.norm(X[:, 1:] - Xr[:, 1:], axis=0) / np.linalg.norm(Xr[:, 1:], axis=0)
    assert err.max() < 1e-10, err


@pytest.mark.parametrize("n", [1, 7, 256, 300, 700])
def test_symmetric_random_uses_ldlt(ctx, n):
    rng = np.random.default_rng(n)
    A = _cplx(rng, n, n)
    Z = A + A.T + 4 * np.sqrt(n) * np.eye(n)   # complex symmetric, well conditioned
    B = _cplx(rng, n, 5)
    X, st = _solve(ctx, Z, B)
    assert st["factorization"] == 1 and st["converged"]
    assert rel(X, np.linalg.solve(Z, B)) < 1e-11


def test_zero_pivot_falls_back_to_lu(ctx):
    rng = np.random.default_rng(2)
    n = 300
    A = _cplx(rng, n, n)
    Z = A + A.T
    Z[0, 0] = 0.0                               # no pivoting cannot start
    B = _cplx(rng, n, 3)
    X, st = _solve(ctx, Z, B)
    assert st["factorization"] == 0 and st["converged"]
    assert rel(X, np.linalg.solve(Z, B)) < 1e-10


def test_hard_symmetric_matrix_still_solves(ctx):
    # an indefinite symmetric matrix with tiny leading pivots: whichever
    # factorisation ends up used, the refined solution is the FP64 one
    rng = np.random.default_rng(9)
    n = 400
    A = _cplx(rng, n, n)
    Z = A + A.T
    Z[:8, :8] *= 1e-6
    B = _cplx(rng, n, 4)
    X, st = _solve(ctx, Z, B)
    assert st["converged"]
    assert rel(X, np.linalg.solve(Z, B)) < 1e-9


def test_nonsymmetric_matrix_uses_lu(ctx):
    rng = np.random.default_rng(4)
    n = 257
    Z = _cplx(rng, n, n) + 10 * np.eye(n)
    B = _cplx(rng, n, 2)
    X, st = _solve(ctx, Z, B)
    assert st["factorization"] == 0
    assert rel(X, np.linalg.solve(Z, B)) < 1e-11
