"""Adjoint gradient of the orientation-averaged M11 misfit with respect to the
refractive index (bem_adjoint_grad), against central differences of the
forward path, and its forward Mueller matrix against bem_dense_run."""
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


@pytest.mark.parametrize("mesh,ka,m", [("ico", 1.5, complex(1.35, 0.02)), ("hex", 2.0, complex(1.5, 0.001))])
def test_gradient_matches_central_differences(ctx, mesh, ka, m):
    import bem_b200 as bb
    v, t = bb.icosphere(1.0, 1) if mesh == "ico" else bb.hex_prism(1.2, 1)
    nt = 19
    # target: the sphere-like reference curve the C5 loss uses, here a fixed smooth curve
    theta = np.linspace(0, np.pi, nt)
    target = 0.05 * (1 + np.cos(theta) ** 2)
    wt = np.linspace(0.5, 1.5, nt)
    kw = dict(orient=(3, 2, 1))
    loss, grad, M = bb.adjoint_grad(ctx, v, t, ka, m, target, wt, **kw)
    assert loss > 0
    h = 1e-5
    fd = []
    for dm in (h, 1j * h):
        lp, _, _ = bb.adjoint_grad(ctx, v, t, ka, m + dm, target, wt, **kw)
        lm, _, _ = bb.adjoint_grad(ctx, v, t, ka, m - dm, target, wt, **kw)
        fd.append((lp - lm) / (2 * h))
    fd = np.array(fd)
    assert np.abs(grad - fd).max() <= 1e-5 * np.abs(fd).max() + 1e-12, (grad, fd)
    # the forward Mueller matrix is the dense pipeline's (FP64)
    M2, _ = bb.dense_run(ctx, v, t, ka, m, orient=(3, 2, 1), ntheta=nt)
    assert rel(M, M2) < 1e-12


def test_zero_misfit_has_zero_gradient(ctx):
    import bem_b200 as bb
    v, t = bb.icosphere(1.0, 1)
    nt = 13
    M, _ = bb.dense_run(ctx, v, t, 1.0, 1.4, orient=(2, 2, 1), ntheta=nt)
    loss, grad, _ = bb.adjoint_grad(ctx, v, t, 1.0, 1.4, M[0, 0], orient=(2, 2, 1))
    assert loss < 1e-28
    assert np.abs(grad).max() < 1e-12


def test_vertex_gradient_matches_central_differences(ctx):
    import bem_b200 as bb
    v, t = bb.c5_mesh(3, refinements=1, rms=0.05)
    nt = 13
    theta = np.linspace(0, np.pi, nt)
    target = 0.04 * (1 + np.cos(theta) ** 2)
    kw = dict(orient=(2, 2, 1))
    ka, m = 1.5, complex(1.33, 0.01)
    loss, grad, M = bb.adjoint_grad_vertices(ctx, v, t, ka, m, target, **kw)
    assert grad.shape == v.shape and np.all(np.isfinite(grad))
    l2, _, M2 = bb.adjoint_grad(ctx, v, t, ka, m, target, **kw)
    assert abs(loss - l2) <= 1e-15 * abs(loss) and np.array_equal(M, M2)
    rng = np.random.default_rng(0)
    h = 1e-5
    scale = np.abs(grad).max()
    for _ in range(4):
        i, c = int(rng.integers(len(v))), int(rng.integers(3))
        lp = bb.adjoint_grad(ctx, v + h * np.eye(1, v.size, 3 * i + c).reshape(v.shape), t, ka, m, target,
                             **kw)[0]
        lm = bb.adjoint_grad(ctx, v - h * np.eye(1, v.size, 3 * i + c).reshape(v.shape), t, ka, m, target,
                             **kw)[0]
        fd = (lp - lm) / (2 * h)
        assert abs(grad[i, c] - fd) <= 1e-5 * scale, (i, c, grad[i, c], fd)
    # a rigid translation changes only phases common to the incident and the
    # scattered field: the orientation-averaged M11 (and the misfit) is invariant
    assert np.abs(grad.sum(axis=0)).max() <= 1e-6 * scale
