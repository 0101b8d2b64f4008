"""Pins the oracle's GMRES (the reference's dense iterative solves,
bem_core.py:1071-1183) against the dependency the reference calls,
scipy.sparse.linalg.gmres, and against the reference's own solutions of the
C1 system (tests/golden/c1_gmres.npz, made by running bem_core.py)."""
import numpy as np
import pytest

from conftest import golden_rwg, load_golden, rel
from oracle import bem_oracle as bo


@pytest.mark.parametrize("n,restart,tol,pc", [(50, 20, 1e-8, "diag"), (120, 10, 1e-6, None),
                                              (80, 5, 1e-10, "diag"), (64, 64, 1e-12, None)])
def test_restatement_replays_scipy(n, restart, tol, pc):
    from scipy.sparse.linalg import LinearOperator, gmres
    rng = np.random.default_rng(n + restart)
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)) + 3 * np.sqrt(n) * np.eye(n)
    b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    ps = bo.precond_solver(A, pc)
    cnt = [0]
    xs, info = gmres(A, b, M=LinearOperator((n, n), matvec=ps, dtype=complex), rtol=tol,
                     restart=restart, maxiter=100, callback_type="pr_norm",
                     callback=lambda r: cnt.__setitem__(0, cnt[0] + 1))
    xo, io, it = bo.gmres(A, b, ps, tol, restart, 100)
    assert (io, it) == (info, cnt[0])
    assert rel(xo, xs) < 1e-13


def test_restatement_maxiter_and_zero_rhs():
    from scipy.sparse.linalg import gmres
    rng = np.random.default_rng(3)
    n = 60
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))   # hard: no shift
    b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    xs, info = gmres(A, b, rtol=1e-12, restart=5, maxiter=3)
    xo, io, it = bo.gmres(A, b, bo.precond_solver(A, None), 1e-12, 5, 3)
    assert info == io == 3 and it == 15
    assert rel(xo, xs) < 1e-12
    x0, i0, it0 = bo.gmres(A, np.zeros(n, complex), bo.precond_solver(A, None), 1e-5, 5, 3)
    assert i0 == 0 and it0 == 0 and not x0.any()


@pytest.fixture(scope="module")
def c1():
    g = load_golden("c1_gmres.npz")
    rwg = golden_rwg(g)
    v, t = g["verts"], g["tris"].astype(np.int64)
    kx, ki, ee, ei = bo.physics(float(g["ka"]), complex(g["m"]))
    Le, Ke = bo.assemble_L_K(rwg, v, t, kx, 7, distance="expanded")
    Li, Ki = bo.assemble_L_K(rwg, v, t, ki, 7, distance="expanded")
    Z = bo.pmchwt_blocks(Le, Ke, Li, Ki, ee, ei)
    return g, Z, bo.aext_matrix(Le, Ke, ee)


def test_aext_preconditioner_reference_solutions(c1):
    g, Z, Aext = c1
    ps = bo.precond_solver(Z, "aext", Aext)
    for c in range(2):
        x, info, it = bo.gmres(Z, g["B"][:, c], ps, float(g["tol_aext"]), min(200, Z.shape[0]),
                               int(g["maxiter_aext"]))
        assert info == 0 and it == g["it_aext"][c]
        assert rel(x, g["x_aext"][:, c]) < 1e-9
        assert np.linalg.norm(g["B"][:, c] - Z @ x) <= float(g["tol_aext"]) * np.linalg.norm(g["B"][:, c])


@pytest.mark.parametrize("tag", ["block_diag", "diag", "none"])
def test_solve_gmres_reference_solutions(c1, tag):
    g, Z, _ = c1
    ps = bo.precond_solver(Z, None if tag == "none" else tag)
    x, info, it = bo.gmres(Z, g["B"][:, 0], ps, float(g["tol"]), 20, int(g["maxiter"]))
    assert info == 0 and bool(g[f"conv_{tag}"])
    assert it == int(g[f"it_{tag}"])
    assert rel(x, g[f"x_{tag}"]) < 1e-8
