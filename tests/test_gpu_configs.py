"""The C2 configuration of the dense path on the device: hex prism aspect
1.4286, refinement 3 (2N = 4608, the reference mesher's size), ka = 5,
m = 1.3116, 8 x 8 x 1 orientations x 2 polarisations = 128 right-hand sides.
The FP64 device LU against SciPy's LAPACK LU of the same device-assembled Z
(lu_solve_full, solver.cu:87-142 / bem_core.py:1637, 1713), and the FP32
factors + FP64 refinement against the FP64 solution at the metric's bar:
1e-9 per column and the orientation-averaged Mueller matrix to 1e-6."""
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


def test_c2_fp64_lapack_and_fp32_refine_bar(ctx):
    from scipy.linalg import lu_factor, lu_solve
    import bem_b200 as bb
    v, t = bb.hex_prism(1.4286, 3)
    g = bb.Geometry(ctx, v, t, 7)
    assert g.n == 4608
    kx, ki, ee, ei = bb.physics(5.0, 1.3116)
    Z = bb.assemble_pmchwt_dev(g, kx, ki, ee, ei)
    RT, w = bb.generate_orientations(8, 8, 1)
    B = bb.rhs_planewave_dev(g, kx, ee, RT)                 # (128, n)
    assert B.shape[0] == 128
    Zh, Bh = Z.cpu().numpy(), B.cpu().numpy()

    lu64 = bb.LU(ctx, Z.clone(), bb.PREC_FP64)
    X64, _ = lu64.solve(B)
    lu64.close()
    lu32 = bb.LU(ctx, Z, bb.PREC_FP32_REFINE)
    X32, st = lu32.solve(B, tol=2e-10, max_iter=12)
    lu32.close()
    assert st["converged"] == 1

    Xr = lu_solve(lu_factor(Zh), Bh.T).T
    X64h, X32h = X64.cpu().numpy(), X32.cpu().numpy()
    col64 = np.linalg.norm(X64h - Xr, axis=1) / np.linalg.norm(Xr, axis=1)
    assert col64.max() < 1e-11, col64.max()
    col32 = np.linalg.norm(X32h - X64h, axis=1) / np.linalg.norm(X64h, axis=1)
    assert col32.max() < 1e-9, (col32.max(), st)

    M64 = bb.mueller_from_solutions_dev(g, X64, RT, w, kx, ee, ntheta=181)
    M32 = bb.mueller_from_solutions_dev(g, X32, RT, w, kx, ee, ntheta=181)
    assert rel(M32, M64) < 1e-6
    # the same Mueller matrix through the one-call pipeline (bem_dense_run)
    Mp, info = bb.dense_run(ctx, v, t, 5.0, 1.3116, orient=(8, 8, 1), ntheta=181,
                            precision=bb.PREC_FP32_REFINE, refine_tol=2e-10)
    assert rel(Mp, M64) < 1e-6
    g.close()
