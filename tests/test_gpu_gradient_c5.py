"""The shape-gradient workload at its full configuration, and the adjoint
contraction kernels against the differences of reassembled operators.

Workload (seeded): an icosphere of refinement 3 (642 vertices, 1926
coordinates, 2N = 3840) displaced radially by a Gaussian random field of
real spherical harmonics of degree <= 6 with RMS 5 % of the radius
(bem_b200.c5_mesh), ka = 5, m = 1.5 + 0.01i, 8 x 8 x 1 orientations, and the
loss sum_theta (M11 - M11_sphere)^2 over 181 angles, M11_sphere the
orientation-averaged M11 of the undisplaced icosphere.  One call of
bem_adjoint_grad_vertices gives all 1926 coordinate gradients and one of
bem_adjoint_grad the two refractive-index ones, each from one forward and one
adjoint solve with the operator's derivative contracted on the fly
(grad_geom.cu).  They are compared with central differences of the forward
loss (bem_dense_run, FP64) at h = 1e-6 (coordinates) and 1e-5 (m), at 1e-5 of
the gradient's largest component; the reference has no gradient code."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KA, M, ORIENT, NTHETA = 5.0, complex(1.5, 0.01), (8, 8, 1), 181


@pytest.fixture(scope="module")
def ctx():
    import bem_b200 as bb
    c = bb.Context(0)
    yield c
    c.close()


def _loss(bb, ctx, v, t, m, target):
    M, _ = bb.dense_run(ctx, v, t, KA, m, orient=ORIENT, ntheta=NTHETA)
    return float(np.sum((M[0, 0] - target) ** 2))


def test_c5_gradients_match_central_differences(ctx):
    import time
    import bem_b200 as bb
    v, t = bb.c5_mesh(11, refinements=3, rms=0.05)
    assert v.shape == (642, 3)
    vs, ts = bb.icosphere(1.0, 3)
    Ms, _ = bb.dense_run(ctx, vs, ts, KA, M, orient=ORIENT, ntheta=NTHETA)
    target = Ms[0, 0].copy()
    t0 = time.perf_counter()
    loss, gv, _ = bb.adjoint_grad_vertices(ctx, v, t, KA, M, target, orient=ORIENT)
    t_v = time.perf_counter() - t0
    loss_m, gm, _ = bb.adjoint_grad(ctx, v, t, KA, M, target, orient=ORIENT)
    assert abs(loss - _loss(bb, ctx, v, t, M, target)) <= 1e-12 * loss
    assert abs(loss - loss_m) <= 1e-14 * loss
    print(f"C5: loss {loss:.6e}, vertex gradient of {gv.size} coordinates in {t_v:.3f} s")
    scale = np.abs(gv).max()
    rng = np.random.default_rng(0)
    h = 1e-6
    for _ in range(8):
        i, c = int(rng.integers(len(v))), int(rng.integers(3))
        vp, vm = v.copy(), v.copy()
        vp[i, c] += h
        vm[i, c] -= h
        fd = (_loss(bb, ctx, vp, t, M, target) - _loss(bb, ctx, vm, t, M, target)) / (2 * h)
        assert abs(gv[i, c] - fd) <= 1e-5 * scale, (i, c, gv[i, c], fd)
    hm = 1e-5
    fdm = [(_loss(bb, ctx, v, t, M + d, target) - _loss(bb, ctx, v, t, M - d, target)) / (2 * hm)
           for d in (hm, 1j * hm)]
    assert np.abs(gm - fdm).max() <= 1e-5 * np.abs(fdm).max(), (gm, fdm)
    # a rigid translation leaves the orientation-averaged M11 unchanged
    assert np.abs(gv.sum(axis=0)).max() <= 1e-6 * scale


def test_contraction_kernels_match_reassembly_differences(ctx):
    # gradient_method 0 (default): the contraction kernels; 1: the operator,
    # right-hand sides and far field reassembled at +-1e-6 per coordinate and
    # +-1e-5 in m, contracted with the same adjoint vectors
    import bem_b200 as bb
    v, t = bb.c5_mesh(3, refinements=2, rms=0.05)
    theta = np.linspace(0, np.pi, 19)
    target = 0.04 * (1 + np.cos(theta) ** 2)
    kw = dict(orient=(3, 2, 1))
    ka, m = 2.5, complex(1.45, 0.02)
    try:
        out = {}
        for method in (0, 1):
            bb.set_option(ctx, "gradient_method", method)
            lv, gv, _ = bb.adjoint_grad_vertices(ctx, v, t, ka, m, target, **kw)
            lm, gm, _ = bb.adjoint_grad(ctx, v, t, ka, m, target, **kw)
            out[method] = (lv, gv, gm)
    finally:
        bb.set_option(ctx, "gradient_method", 0)
    assert out[0][0] == out[1][0]
    assert np.abs(out[0][1] - out[1][1]).max() <= 1e-6 * np.abs(out[1][1]).max()
    assert np.abs(out[0][2] - out[1][2]).max() <= 1e-6 * np.abs(out[1][2]).max(), (out[0][2], out[1][2])
