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


def _oracle_loss(v, t, ka, m, target, orient):
    from oracle import bem_oracle as bo
    t64 = np.asarray(t, dtype=np.int64)
    rwg = bo.build_rwg(v, t64, "cpp")
    kx, ki, ee, ei = bo.physics(ka, m)
    Z = bo.assemble_pmchwt(rwg, v, t64, kx, ki, ee, ei, 7)
    Mo, _, _ = bo.orientation_average_mueller(rwg, v, t64, Z, kx, ee, *orient, len(target), 7)
    return float(np.sum((Mo[0, 0] - target) ** 2))


def test_gradients_against_oracle_central_differences(ctx):
    # an FP64 reference independent of the device path: central differences
    # (h = 1e-5 in m, 1e-6 in a coordinate) of the CPU oracle's forward loss
    import bem_b200 as bb
    v, t = bb.c5_mesh(7, refinements=1, rms=0.05)
    ka, m, orient, nt = 1.5, complex(1.4, 0.01), (2, 2, 1), 13
    theta = np.linspace(0, np.pi, nt)
    target = 0.05 * (1 + np.cos(theta) ** 2)
    loss, gm, _ = bb.adjoint_grad(ctx, v, t, ka, m, target, orient=orient)
    loss_v, gv, _ = bb.adjoint_grad_vertices(ctx, v, t, ka, m, target, orient=orient)
    assert abs(_oracle_loss(v, t, ka, m, target, orient) - loss) <= 1e-9 * loss
    h = 1e-5
    fd = [(_oracle_loss(v, t, ka, m + d, target, orient) - _oracle_loss(v, t, ka, m - d, target, orient)) / (2 * h)
          for d in (h, 1j * h)]
    assert np.abs(gm - fd).max() <= 1e-5 * np.abs(fd).max(), (gm, fd)
    hv = 1e-6
    for iv, c in ((3, 0), (17, 2)):
        vp, vm = v.copy(), v.copy()
        vp[iv, c] += hv
        vm[iv, c] -= hv
        fdv = (_oracle_loss(vp, t, ka, m, target, orient) - _oracle_loss(vm, t, ka, m, target, orient)) / (2 * hv)
        assert abs(gv[iv, c] - fdv) <= 1e-5 * np.abs(gv).max(), (iv, c, gv[iv, c], fdv)


def test_torch_autograd_wrapper(ctx):
    import torch
    import bem_b200 as bb
    v, t = bb.c5_mesh(4, refinements=1, rms=0.05)
    nt = 13
    theta = np.linspace(0, np.pi, nt)
    target = 0.04 * (1 + np.cos(theta) ** 2)
    kw = dict(orient=(2, 2, 1))
    verts = torch.tensor(v, dtype=torch.float64, requires_grad=True)
    m_re = torch.tensor(1.45, dtype=torch.float64, requires_grad=True)
    m_im = torch.tensor(0.01, dtype=torch.float64, requires_grad=True)
    loss = bb.mueller_misfit(ctx, verts, t, 2.0, m_re, m_im, target, **kw)
    (3.0 * loss).backward()
    l1, gv, _ = bb.adjoint_grad_vertices(ctx, v, t, 2.0, complex(1.45, 0.01), target, **kw)
    l2, gm, _ = bb.adjoint_grad(ctx, v, t, 2.0, complex(1.45, 0.01), target, **kw)
    assert loss.item() == l1 and abs(l1 - l2) <= 1e-12 * l1
    assert np.array_equal(verts.grad.numpy(), 3.0 * gv)
    assert float(m_re.grad) == 3.0 * gm[0] and float(m_im.grad) == 3.0 * gm[1]
    # vertices without a gradient: only the refractive-index adjoint runs
    m_re.grad = None
    loss2 = bb.mueller_misfit(ctx, torch.tensor(v), t, 2.0, m_re, m_im, target, **kw)
    loss2.backward()
    assert loss2.item() == l2 and float(m_re.grad) == gm[0]
