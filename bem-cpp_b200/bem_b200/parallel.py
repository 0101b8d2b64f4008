"""Multi-GPU plumbing for the dense path: replicas, not a distributed LU.

Every rank assembles and factors its own copy of Z (the factorisation of one
2N x 2N matrix does not shard without a block-cyclic distributed LU); the
orientation x polarisation right-hand sides are split into contiguous slices,
each rank solves its slice and forms its part of the weighted Mueller sum,
and one all-reduce (sum) of the 16 x ntheta partial Mueller matrices gives
the orientation average -- the device-side counterpart of the reference's
--orient-range split with a JSON sum (cluster_bem.py:76-127).  Batches of
particles split the same way: each rank runs its contiguous slice of the
particles and the results are gathered on every rank (cluster_bem.py farms
one process per particle).
"""
from __future__ import annotations

import numpy as np


def orientation_slice(n_orient: int, rank: int, world: int):
    """Contiguous [o0, o1) of orientations for `rank` (sizes differ by <= 1)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank / world size")
    return rank * n_orient // world, (rank + 1) * n_orient // world


def allreduce_sum(x, device=None):
    """Sum a numpy array (e.g. a partial Mueller matrix) over all ranks of the
    default process group; returns a numpy array."""
    import torch
    import torch.distributed as dist
    t = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64))
    if device is not None:
        t = t.to(device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.cpu().numpy()


def allreduce_max(x: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def raise_if_any_rank_failed(err, what):
    """Every rank calls this after its local work, failed or not, so the
    ranks take the same collective: one all_gather_object of the local error
    (None or a message); if any rank failed, every rank raises RuntimeError
    naming the first failed rank, instead of the others waiting in their next
    collective until the process group's timeout."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        errs = [None] * dist.get_world_size()
        dist.all_gather_object(errs, err)
    else:
        errs = [err]
    for r, e in enumerate(errs):
        if e is not None:
            raise RuntimeError(f"{what}: rank {r} failed: {e}")


def orientation_average_distributed(ctx, geom, Z, RT, w, k_ext, eta_ext, ntheta=181,
                                    precision=None, tol=0.0, rank=0, world=1, device=None):
    """Orientation-averaged Mueller matrix with the orientations split across
    ranks.  Z is this rank's full copy of the system matrix (device tensor).
    Returns (M (4,4,ntheta) summed over ranks, this rank's solve stats)."""
    from . import api
    from ._lib import PREC_FP32_REFINE
    if precision is None:
        precision = PREC_FP32_REFINE
    o0, o1 = orientation_slice(len(w), rank, world)
    part = np.zeros((4, 4, ntheta))
    stats, err = None, None
    if o1 > o0:
        try:
            B = api.rhs_planewave_dev(geom, k_ext, eta_ext, RT[o0:o1])
            lu = api.LU(ctx, Z, precision)
            X, stats = lu.solve(B, tol=tol)
            lu.close()
            part = api.mueller_from_solutions_dev(geom, X, RT[o0:o1], w[o0:o1], k_ext, eta_ext, ntheta)
        except Exception as ex:  # the collectives below are taken either way
            err = f"{type(ex).__name__}: {ex}"
    raise_if_any_rank_failed(err, "orientation_average_distributed")
    return allreduce_sum(part, device).reshape(4, 4, ntheta), stats


def particle_slice(count: int, rank: int, world: int):
    """Contiguous [p0, p1) of a batch of `count` particles for `rank`."""
    return orientation_slice(count, rank, world)


def batch_run_distributed(ctx, particles, rank=0, world=1, run=None):
    """Particles split across ranks: rank r runs particle_slice(len, r, world)
    with `run` (default: api.batch_run on this rank's context, no raising),
    then every rank receives all results in particle order through one
    all_gather_object of the default process group.  Returns the list of
    (mueller, info) for every particle."""
    import torch.distributed as dist
    if run is None:
        from . import api

        def run(ps):
            return api.batch_run(ctx, ps, raise_on_error=False)
    p0, p1 = particle_slice(len(particles), rank, world)
    mine, err = [], None
    try:
        mine = list(run(particles[p0:p1])) if p1 > p0 else []
    except Exception as ex:  # the collectives below are taken either way
        err = f"{type(ex).__name__}: {ex}"
    raise_if_any_rank_failed(err, "batch_run_distributed")
    if world <= 1 or not (dist.is_available() and dist.is_initialized()):
        return mine
    parts = [None] * world
    dist.all_gather_object(parts, (p0, mine))
    out = []
    for q0, res in sorted(parts, key=lambda x: x[0]):
        out.extend(res)
    return out
