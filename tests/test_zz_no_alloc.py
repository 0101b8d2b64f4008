"""The allocation-free Mueller entry point (bem_farfield_mueller_noalloc).

It exists for callers that cannot allocate device memory, such as hosts
whose device memory is owned by their own allocator.  Its scratch is a static device
array shared by all calls, so this file checks it against the allocating
entry point (bem_farfield_mueller_dev) over the C ABI on two calls in a row
with different orientation sets: a stale second call would show there.  The
file is named to be collected last."""
import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu


def _problem(bb, ctx):
    import torch
    v, t = bb.icosphere(1.0, 1)
    g = bb.Geometry(ctx, v, t, 7)
    kx, ki, ee, ei = bb.physics(2.0, 1.3116 + 0.01j)
    Z = bb.assemble_pmchwt_dev(g, kx, ki, ee, ei)
    RT, w = bb.generate_orientations(3, 3, 1)
    B = bb.rhs_planewave_dev(g, kx, ee, RT)
    lu = bb.LU(ctx, Z, bb.PREC_FP64)
    X, _ = lu.solve(B)
    torch.cuda.synchronize()
    return g, X, RT, w, kx, ee


def test_noalloc_matches_allocating_entry_point_twice():
    import torch
    import bem_b200 as bb
    ctx = bb.Context(0)
    g, X, RT, w, kx, ee = _problem(bb, ctx)
    nt = 37
    # call 1: all 9 orientations; call 2: a different subset (3 orientations)
    cases = [(slice(0, 9), False), (slice(2, 5), True)]
    for sl, mirror in cases:
        Xs = X[2 * sl.start:2 * sl.stop]
        M_ref = bb.mueller_from_solutions_dev(g, Xs, RT[sl], w[sl], kx, ee, ntheta=nt,
                                              gamma_mirror=mirror)
        M_out = torch.full((16 * nt,), float("nan"), dtype=torch.float64, device="cuda")
        bb.mueller_noalloc_dev(g, Xs, RT[sl], w[sl], kx, ee, M_out, ntheta=nt, gamma_mirror=mirror)
        torch.cuda.synchronize()
        M = M_out.cpu().numpy().reshape(4, 4, nt)
        assert np.all(np.isfinite(M))
        assert rel(M, M_ref) < 1e-13


def test_noalloc_rejects_oversized_request():
    import torch
    import bem_b200 as bb
    ctx = bb.Context(0)
    g, X, RT, w, kx, ee = _problem(bb, ctx)
    # 9 orientations x 4000 angles x 16 doubles = 4.6 MB > 4 MiB
    M_out = torch.zeros(16 * 4000, dtype=torch.float64, device="cuda")
    with pytest.raises(bb.BemError) as e:
        bb.mueller_noalloc_dev(g, X, RT, w, kx, ee, M_out, ntheta=4000)
    assert e.value.status == 1 and "maximum" in str(e.value)
