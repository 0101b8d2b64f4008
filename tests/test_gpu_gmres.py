"""GMRES on the dense Z (bem_core.py:1071-1183): the device A_ext, the batched
device GMRES against the oracle's restatement of scipy's gmres on the same
device-assembled Z (iteration counts equal per column), and against the
reference's own solutions of the C1 system (tests/golden/c1_gmres.npz)."""
import numpy as np
import pytest

from conftest import golden_rwg, load_golden, rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import bem_b200 as bb
    c = bb.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def c1(ctx):
    """The C1 system in the reference's RWG order: device Z, the golden."""
    import bem_b200 as bb
    g = load_golden("c1_gmres.npz")
    geom = bb.Geometry.from_rwg(ctx, g["verts"], g["tris"], golden_rwg(g), 7)
    kx, ki, ee, ei = bb.physics(float(g["ka"]), complex(g["m"]))
    Z = bb.assemble_pmchwt_dev(geom, kx, ki, ee, ei)
    yield g, geom, Z, (kx, ee)
    geom.close()


def test_aext_matrix_matches_oracle(ctx):
    import bem_b200 as bb
    from oracle import bem_oracle as bo
    v, t = bb.icosphere(1.0, 1)
    geom = bb.Geometry(ctx, v, t, 7)
    kx, _, ee, _ = bb.physics(2.0, 1.4)
    A = bb.assemble_aext_dev(geom, kx, ee).cpu().numpy()
    rwg = bo.build_rwg(v, t.astype(np.int64), "cpp")
    Le, Ke = bo.assemble_L_K(rwg, v, t.astype(np.int64), kx, 7)
    assert rel(A, bo.aext_matrix(Le, Ke, ee)) < 1e-12
    # the exterior part of the full PMCHWT: Z - A_ext holds only the interior medium
    Lx, Kx = bb.assemble_L_K_dev(geom, kx)
    N = geom.N
    assert rel(A[N:, :N], Kx.cpu().numpy()) < 1e-15
    geom.close()


def test_aext_gmres_reference_solutions(ctx, c1):
    import bem_b200 as bb
    g, geom, Z, (kx, ee) = c1
    M, _ = bb.build_aext_preconditioner(geom, kx, ee)
    X, info = bb.gmres(ctx, Z, g["B"], M, tol=float(g["tol_aext"]), restart=min(200, geom.n),
                       maxiter=int(g["maxiter_aext"]))
    M.close()
    assert list(info["iters"]) == list(g["it_aext"]) and not info["info"].any()
    # the device Z differs from the reference's by its distance-expansion noise
    assert rel(X, g["x_aext"]) < 1e-6
    Zh = Z.cpu().numpy()
    for c in range(2):
        assert np.linalg.norm(g["B"][:, c] - Zh @ X[:, c]) <= float(g["tol_aext"]) * np.linalg.norm(g["B"][:, c])


@pytest.mark.parametrize("tag", ["block_diag", "diag", "none"])
def test_solve_gmres_reference_solutions(ctx, c1, tag):
    import bem_b200 as bb
    from oracle import bem_oracle as bo
    g, geom, Z, _ = c1
    b = g["B"][:, 0]
    pc = None if tag == "none" else tag
    x = bb.solve_gmres(ctx, Z, b, tol=float(g["tol"]), maxiter=int(g["maxiter"]), precond=pc)
    assert rel(x, g[f"x_{tag}"]) < 1e-5
    # the same algorithm on the same device Z: the oracle's restatement
    Zh = Z.cpu().numpy()
    xo, io, it = bo.gmres(Zh, b, bo.precond_solver(Zh, pc), float(g["tol"]), 20, int(g["maxiter"]))
    M = bb.Preconditioner(ctx, pc, Z=Z)
    _, info = bb.gmres(ctx, Z, b, M, tol=float(g["tol"]), restart=20, maxiter=int(g["maxiter"]))
    M.close()
    assert (int(info["iters"][0]), int(info["info"][0])) == (it, io) == (int(g[f"it_{tag}"]), 0)
    assert rel(x, xo) < 1e-9


def test_batched_columns_replay_the_oracle(ctx):
    import bem_b200 as bb
    from oracle import bem_oracle as bo
    v, t = bb.icosphere(1.0, 2)
    geom = bb.Geometry(ctx, v, t, 7)
    kx, ki, ee, ei = bb.physics(3.0, complex(1.5, 0.01))
    Z = bb.assemble_pmchwt_dev(geom, kx, ki, ee, ei)
    RT, _ = bb.generate_orientations(3, 3, 1)
    B = bb.rhs_planewave_dev(geom, kx, ee, RT)             # (18, n): 9 orientations x 2
    B[5].zero_()                                            # a zero right-hand side
    M = bb.Preconditioner(ctx, "diag", Z=Z)
    X, info = bb.gmres(ctx, Z, B, M, tol=1e-7, restart=15, maxiter=50)
    M.close()
    Zh, Bh, Xh = Z.cpu().numpy(), B.cpu().numpy(), X.cpu().numpy()
    ps = bo.precond_solver(Zh, "diag")
    for c in range(Bh.shape[0]):
        xo, io, it = bo.gmres(Zh, Bh[c], ps, 1e-7, 15, 50)
        assert (int(info["iters"][c]), int(info["info"][c])) == (it, io), c
        if c == 5:
            assert it == 0 and not Xh[c].any()
        else:
            assert rel(Xh[c], xo) < 1e-10, c
    assert info["converged"] == 1 and info["max_rel_residual"] <= 1e-7
    geom.close()


def test_maxiter_and_restart_cycles_replay_the_oracle(ctx, c1):
    import bem_b200 as bb
    from oracle import bem_oracle as bo
    g, geom, Z, _ = c1
    b = g["B"][:, 1]
    X, info = bb.gmres(ctx, Z, b, None, tol=1e-9, restart=6, maxiter=4)
    Zh = Z.cpu().numpy()
    xo, io, it = bo.gmres(Zh, b, bo.precond_solver(Zh, None), 1e-9, 6, 4)
    assert io == 4 and (int(info["iters"][0]), int(info["info"][0])) == (it, io)
    assert info["converged"] == 0 and info["n_unconverged"] == 1 and info["max_cycles"] == 4
    assert rel(X, xo) < 1e-10


def test_fp32_preconditioners_reach_the_tolerance(ctx, c1):
    import bem_b200 as bb
    g, geom, Z, (kx, ee) = c1
    Zh = Z.cpu().numpy()
    M, _ = bb.build_aext_preconditioner(geom, kx, ee, precision=bb.PREC_FP32_REFINE)
    X, info = bb.gmres(ctx, Z, g["B"], M, tol=1e-10, restart=200, maxiter=20)
    M.close()
    # FP32 factors: a slightly inexact preconditioner (25 inner iterations
    # measured at 2N = 960 against 7 to reach 1e-5 with FP64 factors)
    assert info["converged"] == 1 and info["max_iterations"] <= 40
    for c in range(2):
        assert np.linalg.norm(g["B"][:, c] - Zh @ X[:, c]) <= 1e-10 * np.linalg.norm(g["B"][:, c])
    x = bb.solve_gmres(ctx, Z, g["B"][:, 0], tol=1e-8, precond="block_diag", precision=bb.PREC_FP32_REFINE)
    assert np.linalg.norm(g["B"][:, 0] - Zh @ x) <= 1e-8 * np.linalg.norm(g["B"][:, 0])


def test_int8_products_agree_with_fp64(ctx, c1):
    import bem_b200 as bb
    g, geom, Z, (kx, ee) = c1
    M, _ = bb.build_aext_preconditioner(geom, kx, ee)
    X64, i64 = bb.gmres(ctx, Z, g["B"], M, tol=1e-10, restart=50, maxiter=10)
    bb.set_option(ctx, "gmres_digits", 7)
    try:
        X8, i8 = bb.gmres(ctx, Z, g["B"], M, tol=1e-10, restart=50, maxiter=10)
    finally:
        bb.set_option(ctx, "gmres_digits", 0)
    M.close()
    assert list(i8["iters"]) == list(i64["iters"])
    assert rel(X8, X64) < 1e-11


def test_bad_arguments(ctx, c1):
    import torch
    import bem_b200 as bb
    g, geom, Z, _ = c1
    B = torch.from_numpy(np.ascontiguousarray(g["B"].T)).cuda()
    M = bb.Preconditioner(ctx, None, n=geom.n)
    with pytest.raises(bb.BemError):                        # X aliasing B
        ctx.check(bb.lib().bem_gmres_solve_dev(
            ctx.h, Z.data_ptr(), geom.n, geom.n, M.h, B.data_ptr(), geom.n, B.data_ptr(), geom.n,
            2, 20, 1e-5, 10, None, None, None))
    M.close()
    Zodd = torch.zeros((5, 5), dtype=torch.complex128, device="cuda")
    with pytest.raises(bb.BemError):
        bb.Preconditioner(ctx, "block_diag", Z=Zodd)
    with pytest.raises(bb.BemError):
        bb.Preconditioner(ctx, "diag", Z=Zodd)              # zero diagonal
    with pytest.raises(bb.BemError):
        bb.gmres(ctx, Z, g["B"], bb.Preconditioner(ctx, None, n=4))   # order mismatch


def test_dense_run_with_gmres_aext(ctx):
    # orientation averaging solved column by column with GMRES(A_ext), as the
    # reference's orientation functions do when given Z_ext_lu
    # (bem_core.py:1703-1709): the Mueller matrix agrees with the LU path to
    # the GMRES tolerance
    import bem_b200 as bb
    v, t = bb.icosphere(1.0, 2)
    kw = dict(orient=(3, 4, 1), ntheta=37)
    M_lu, _ = bb.dense_run(ctx, v, t, 2.0, complex(1.4, 0.01), **kw)
    M_gm, info = bb.dense_run(ctx, v, t, 2.0, complex(1.4, 0.01), solver="gmres_aext", gmres_tol=1e-8, **kw)
    g = info["gmres"]
    assert g["converged"] == 1 and g["n_unconverged"] == 0 and 0 < g["max_iterations"] <= 30
    assert g["max_rel_residual"] <= 1e-8
    assert rel(M_gm, M_lu) < 1e-6
    M32, i32 = bb.dense_run(ctx, v, t, 2.0, complex(1.4, 0.01), solver="gmres_aext", gmres_tol=1e-8,
                            precision=bb.PREC_FP32_REFINE, **kw)
    assert i32["gmres"]["converged"] == 1 and rel(M32, M_lu) < 1e-6


def test_cli_dense_solver_gmres_aext(tmp_path):
    import json
    import os
    import subprocess
    cli = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "bem-cpp_b200", "bin",
                       "bem_cuda")
    if not os.path.exists(cli):
        pytest.skip("bem_cuda not built")
    base = [cli, "--ka", "1.5", "--ref", "2", "--ri", "1.33", "0.0", "--orient", "2", "3", "1", "--ntheta", "19"]
    out = {}
    for tag, extra in (("lu", []), ("gm", ["--dense-solver", "gmres-aext", "--gmres-tol", "1e-9"])):
        f = tmp_path / f"{tag}.json"
        run = subprocess.run(base + extra + ["--out", str(f)], check=True, capture_output=True, text=True,
                             timeout=300)
        out[tag] = (np.array(json.loads(f.read_text())["mueller"]), run.stdout)
    assert "GMRES(A_ext)" in out["gm"][1]
    assert rel(out["gm"][0], out["lu"][0]) < 1e-6
