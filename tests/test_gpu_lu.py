"""Device LU / multi-RHS solve against LAPACK (scipy) on the same matrices."""
import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import bem_b200 as bb
    c = bb.Context(0)
    yield c
    c.close()


def _rand(n, seed, cond_boost=True):
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    return A


@pytest.mark.parametrize("n,nrhs", [(1, 1), (5, 3), (17, 2), (257, 7), (300, 33), (1000, 64)])
def test_fp64_random_against_numpy(ctx, n, nrhs):
    import torch
    import bem_b200 as bb
    A = _rand(n, n)
    B = _rand(max(n, nrhs), n + 1)[:n, :nrhs]
    Zt = torch.from_numpy(A.copy()).cuda()
    lu = bb.LU(ctx, Zt, bb.PREC_FP64)
    assert lu.info == 0
    X, _ = lu.solve(B)
    Xr = np.linalg.solve(A, B)
    assert rel(X.cpu().numpy().T, Xr) < 1e-11


def test_pivot_sequence_matches_lapack(ctx):
    # izamax rule (max |re|+|im|, first index) on a matrix without ties
    from scipy.linalg import lu_factor
    import bem_b200 as bb
    A = _rand(200, 3)
    F, ipiv, info = bb.lu_factorize_cuda(ctx, A)
    lu_t, piv_t = lu_factor(A.T)  # row-major A seen as column-major A^T: LAPACK pivots rows of A^T
    # our P A = L U with row pivots of A; compare against LAPACK on A itself
    lu2, piv2 = lu_factor(A)
    assert info == 0
    assert np.array_equal(ipiv - 1, piv2)
    assert rel(F, lu2) < 1e-12


@pytest.mark.parametrize("n", [700, 1500])
def test_fp64_gemm_3m_against_4m(ctx, n):
    # the FP64 trailing updates and solves with three real products per
    # complex one (default) against four: the same pivots (LAPACK's), and
    # backward errors of the factors and of the solutions within a small
    # factor of the four-product ones (3M's normwise bound is ~1.3x larger
    # in a NumPy emulation of this blocked LU; forward errors of random
    # matrices scatter by several times either way, so they are not compared)
    import bem_b200 as bb
    from scipy.linalg import lu_factor
    A = _rand(n, 40 + n)
    B = _rand(n, 41 + n)[:, :24]
    out = {}
    try:
        for m3 in (1, 0):
            bb.set_option(ctx, "fp64_gemm_3m", m3)
            F, ipiv, info = bb.lu_factorize_cuda(ctx, A)
            assert info == 0
            out[m3] = (F, ipiv, bb.lu_solve_cuda(ctx, F, ipiv, B))
    finally:
        bb.set_option(ctx, "fp64_gemm_3m", 1)
    _, piv2 = lu_factor(A)
    assert np.array_equal(out[1][1], out[0][1])
    assert np.array_equal(out[1][1] - 1, piv2)
    nA = np.linalg.norm(A)

    def factor_backward(F, ipiv):
        PA = A.copy()
        for i, p in enumerate(ipiv - 1):  # LAPACK row interchanges, in order
            PA[[i, p]] = PA[[p, i]]
        L = np.tril(F, -1) + np.eye(n)
        return np.linalg.norm(PA - L @ np.triu(F)) / nA

    def solve_backward(X):
        return np.linalg.norm(A @ X - B) / (nA * np.linalg.norm(X))

    f3, f4 = factor_backward(*out[1][:2]), factor_backward(*out[0][:2])
    s3, s4 = solve_backward(out[1][2]), solve_backward(out[0][2])
    # (measured: f4 1.2e-14 / 2.5e-14, f3 1.8e-14 / 4.1e-14 at n = 700 / 1500)
    assert f3 < 1e-16 * n and f3 <= 2 * f4, (f3, f4)
    assert s3 < 1e-16 * n and s3 <= 2 * s4, (s3, s4)
    assert rel(out[1][2], np.linalg.solve(A, B)) < 1e-10


@pytest.mark.parametrize("n", [600, 1300])
def test_fp64_u12_slabs_against_triangular_solve(ctx, n):
    # lu_u12_slabs (default): U12 = L11^-1 A12 by 64-row slabs with GEMM
    # updates between them; 0: one block triangular solve.  Same pivots
    # (LAPACK's), backward errors of the factors and solutions within a small
    # factor of each other
    import bem_b200 as bb
    from scipy.linalg import lu_factor
    A = _rand(n, 70 + n)
    B = _rand(n, 71 + n)[:, :12]
    out = {}
    try:
        for inv in (1, 0):
            bb.set_option(ctx, "lu_u12_slabs", inv)
            F, ipiv, info = bb.lu_factorize_cuda(ctx, A)
            assert info == 0
            out[inv] = (F, ipiv, bb.lu_solve_cuda(ctx, F, ipiv, B))
    finally:
        bb.set_option(ctx, "lu_u12_slabs", 1)
    _, piv2 = lu_factor(A)
    assert np.array_equal(out[1][1], out[0][1])
    assert np.array_equal(out[1][1] - 1, piv2)
    nA = np.linalg.norm(A)
    fb = []
    for F, ipiv, X in out.values():
        PA = A.copy()
        for i, p in enumerate(ipiv - 1):
            PA[[i, p]] = PA[[p, i]]
        fb.append(np.linalg.norm(PA - (np.tril(F, -1) + np.eye(n)) @ np.triu(F)) / nA)
        assert np.linalg.norm(A @ X - B) / (nA * np.linalg.norm(X)) < 1e-16 * n
    assert fb[0] < 1e-16 * n and fb[0] <= 3 * fb[1], fb


def test_singular_reports_info(ctx):
    import bem_b200 as bb
    A = _rand(64, 4)
    A[:, 10] = 0.0
    F, ipiv, info = bb.lu_factorize_cuda(ctx, A)
    assert info == 11


def test_host_mirrors_round_trip(ctx):
    import bem_b200 as bb
    A = _rand(300, 5)
    B = _rand(300, 6)[:, :9]
    F, ipiv, info = bb.lu_factorize_cuda(ctx, A)
    X = bb.lu_solve_cuda(ctx, F, ipiv, B)
    assert rel(X, np.linalg.solve(A, B)) < 1e-11
    X2, st = bb.lu_solve_full(ctx, A, B, bb.PREC_FP64)
    assert rel(X2, np.linalg.solve(A, B)) < 1e-11


@pytest.mark.parametrize("n,nrhs", [(600, 16), (1100, 40)])
def test_fp32_refine_reaches_fp64(ctx, n, nrhs):
    import torch
    import bem_b200 as bb
    A = _rand(n, 7) + 4 * np.sqrt(n) * np.eye(n)
    B = _rand(max(n, nrhs), 8)[:n, :nrhs]
    Zt = torch.from_numpy(A.copy()).cuda()
    lu = bb.LU(ctx, Zt, bb.PREC_FP32_REFINE)
    X, st = lu.solve(B, tol=1e-13)
    Xr = np.linalg.solve(A, B)
    Xn = X.cpu().numpy().T
    err = np.max(np.linalg.norm(Xn - Xr, axis=0) / np.linalg.norm(Xr, axis=0))
    assert st["converged"] == 1 and err < 1e-10, (st, err)


def test_pmchwt_fp64_and_fp32_refine(ctx):
    # assembled ico ref 2 system (n=960): FP64 vs LAPACK; FP32+refine vs FP64 at 1e-9
    import torch
    import bem_b200 as bb
    from scipy.linalg import lu_factor, lu_solve
    v, t = bb.icosphere(1.0, 2)
    g = bb.Geometry(ctx, v, t, 7)
    kx, ki, ee, ei = bb.physics(1.0, 1.3116)
    Z = bb.assemble_pmchwt_dev(g, kx, ki, ee, ei)
    Zh = Z.cpu().numpy()
    rng = np.random.default_rng(11)
    B = rng.standard_normal((g.n, 6)) + 1j * rng.standard_normal((g.n, 6))
    Xr = lu_solve(lu_factor(Zh), B)
    lu32 = bb.LU(ctx, Z, bb.PREC_FP32_REFINE)
    X32, st = lu32.solve(B, tol=1e-12)
    lu64 = bb.LU(ctx, Z.clone(), bb.PREC_FP64)
    X64, _ = lu64.solve(B)
    X64 = X64.cpu().numpy().T
    X32 = X32.cpu().numpy().T
    assert rel(X64, Xr) < 1e-12
    col = np.linalg.norm(X32 - X64, axis=0) / np.linalg.norm(X64, axis=0)
    assert col.max() < 1e-9, (col.max(), st)


def test_factor_memory_cache_reuses_blocks_bitwise(ctx):
    # cache_factor_memory: a loop of factorisations of one order reuses the
    # FP32 factor and digit-plane blocks; results are bitwise those of fresh
    # allocations, and switching the option off returns the memory
    import torch
    import bem_b200 as bb
    rng = np.random.default_rng(17)
    n = 640
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)) + 4 * np.sqrt(n) * np.eye(n)
    Z = torch.from_numpy(A).cuda()
    B = torch.from_numpy(np.ascontiguousarray((rng.standard_normal((n, 6)) + 0j).T)).cuda()

    def run():
        lu = bb.LU(ctx, Z, bb.PREC_FP32_REFINE)
        X, st = lu.solve(B, tol=1e-12)
        lu.close()
        torch.cuda.synchronize()
        return X.cpu().numpy(), st

    X0, _ = run()
    bb.set_option(ctx, "cache_factor_memory", 1)
    try:
        free0 = torch.cuda.mem_get_info()[0]
        X1, _ = run()
        held = free0 - torch.cuda.mem_get_info()[0]
        X2, _ = run()
        assert held >= n * n * 8                     # the FP32 factors stay allocated
        assert free0 - torch.cuda.mem_get_info()[0] <= held + (2 << 20)   # and are reused
    finally:
        bb.set_option(ctx, "cache_factor_memory", 0)
    assert torch.cuda.mem_get_info()[0] >= free0 - (2 << 20)
    assert np.array_equal(X0, X1) and np.array_equal(X1, X2)


@pytest.mark.parametrize("n", [40, 700, 2000, 4608, 7000])
def test_cluster_panels_match_grid_panels(ctx, n):
    # the sub-panels on thread-block clusters (default: every sub-panel of
    # up to ~5700 rows) against the cooperative grid kernel: the same pivot
    # rule and per-element arithmetic (explicit FMAs), so bitwise the same
    # pivots and factors; at
    # n = 7000 the first sub-panels are too tall for a cluster and the two
    # kernels alternate within one factorisation
    import bem_b200 as bb
    A = _rand(n, 10 + n)
    A[:, 5] = 0.0  # a zero pivot on the way: info and the skipped scaling
    out = {}
    try:
        for mode in (1, 0):
            bb.set_option(ctx, "panel_clusters", mode)
            out[mode] = bb.lu_factorize_cuda(ctx, A)
    finally:
        bb.set_option(ctx, "panel_clusters", 1)
    (F1, p1, i1), (F0, p0, i0) = out[1], out[0]
    assert i1 == i0 == 6
    assert np.array_equal(p1, p0)
    assert np.array_equal(F1, F0)


def test_cluster_panels_batched(ctx):
    # batched factorisation (one cluster per matrix in one launch) against
    # the single LU of each matrix
    import bem_b200 as bb
    parts = bb.c4_particles(seed=5, count=3, ntheta=19)
    single = [bb.dense_run(ctx, **{k: v for k, v in p.items() if k != "meta"})[0] for p in parts]
    try:
        bb.set_option(ctx, "lu_autotune", 0)
        out = bb.batch_run(ctx, parts)
    finally:
        bb.set_option(ctx, "lu_autotune", 1)
    for M1, (M, info) in zip(single, out):
        assert info["status"] == 0 and np.array_equal(M, M1)
