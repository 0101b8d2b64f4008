"""Failure detection on the device without a fault: a bounded wait on a flag
that nothing sets runs out, the call returns BEM_ERR_TIMEOUT, and the same
context then runs a solve (bem_selftest_bounded_wait runs the wait pattern
of the library's kernels alone)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_bounded_wait_runs_out_and_the_context_stays_usable():
    import torch
    import bem_b200 as bb
    ctx = bb.Context(0)
    L = bb.lib()
    with pytest.raises(bb.BemError) as ei:
        ctx.check(L.bem_selftest_bounded_wait(ctx.h, 2_000_000, 0))      # ~1 ms of clock cycles
    assert ei.value.status == 6 and "ran out" in str(ei.value)
    ctx.check(L.bem_selftest_bounded_wait(ctx.h, 2_000_000, 1))          # the flag is set: no wait
    assert L.bem_selftest_bounded_wait(ctx.h, -1, 0) == 1                  # BEM_ERR_INVALID
    rng = np.random.default_rng(0)
    n = 300
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)) + 3 * np.sqrt(n) * np.eye(n)
    B = rng.standard_normal((n, 3)) + 0j
    lu = bb.LU(ctx, torch.from_numpy(A).cuda(), bb.PREC_FP64)
    X, _ = lu.solve(torch.from_numpy(np.ascontiguousarray(B.T)).cuda())
    lu.close()
    assert np.abs(A @ X.cpu().numpy().T - B).max() < 1e-10
    ctx.close()
