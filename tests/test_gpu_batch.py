"""Batched particles (bem_batch_run): the seeded hex-prism workload.  FP64
particles of one system size run as a bucket (one assembly pass, one batched
LU and one batched solve per size): with the single LU's block shape every
particle is bitwise its own bem_dense_run, with the autotuned shape within
rounding of it; one particle against the oracle; FP32 + refinement against
FP64 per particle; and a failing particle that does not stop the batch."""
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


def test_batch_equals_individual_runs(ctx):
    import bem_b200 as bb
    parts = bb.c4_particles(seed=5, count=6, ntheta=37)
    sizes = [p["meta"]["refinements"] for p in parts]
    assert min(sizes.count(2), sizes.count(3)) >= 2, "seed 5 draws three of each size: both buckets batched"
    ref = []
    for p in parts:
        kw = {k: v for k, v in p.items() if k != "meta"}
        ref.append(bb.dense_run(ctx, **kw)[0])
    try:
        bb.set_option(ctx, "lu_autotune", 0)  # the single LU's shape: bitwise the same factors
        out = bb.batch_run(ctx, parts)
    finally:
        bb.set_option(ctx, "lu_autotune", 1)
    assert len(out) == 6
    for M1, (M, info) in zip(ref, out):
        assert info["status"] == 0
        assert info["N"] in (576, 2304) and info["n_orient"] == 16
        assert np.array_equal(M, M1)
        assert np.all(np.isfinite(M)) and np.all(M[0, 0] > 0)
    # the autotuned block / panel widths: other rounding, same solution
    out = bb.batch_run(ctx, parts)
    for M1, (M, info) in zip(ref, out):
        assert info["status"] == 0 and rel(M, M1) < 1e-12
    # one at a time (batch_buckets 0) is the dense pipeline itself
    try:
        bb.set_option(ctx, "batch_buckets", 0)
        out = bb.batch_run(ctx, parts[:2])
    finally:
        bb.set_option(ctx, "batch_buckets", 1)
    assert all(np.array_equal(M, M1) for M1, (M, _) in zip(ref, out))


def test_fp32_refine_particles_against_fp64(ctx):
    import bem_b200 as bb
    p64 = bb.c4_particles(seed=4, count=8, ntheta=37)
    p32 = bb.c4_particles(seed=4, count=8, ntheta=37, precision=bb.PREC_FP32_REFINE)
    o64, o32 = bb.batch_run(ctx, p64), bb.batch_run(ctx, p32)
    for (M64, i64), (M32, i32) in zip(o64, o32):
        assert i64["status"] == 0 and i32["status"] == 0
        assert i32["stats"]["converged"] == 1
        assert rel(M32, M64) < 1e-6


def test_batch_particle_against_oracle(ctx):
    import bem_b200 as bb
    from oracle import bem_oracle as bo
    parts = [p for p in bb.c4_particles(seed=11, count=8, ntheta=19)
             if p["meta"]["refinements"] == 2][:1]
    assert parts, "seed 11 draws at least one refinement-2 prism"
    p = parts[0]
    (M, info), = bb.batch_run(ctx, parts)
    v, t = p["verts"], p["tris"].astype(np.int64)
    rwg = bo.build_rwg(v, t, "cpp")
    kx, ki, ee, ei = bo.physics(p["ka"], p["m"])
    Zo = bo.assemble_pmchwt(rwg, v, t, kx, ki, ee, ei, 7)
    Mo, _, _ = bo.orientation_average_mueller(rwg, v, t, Zo, kx, ee, 4, 4, 1, 19, 7)
    assert rel(M, Mo) < 1e-10


def test_failing_particle_does_not_stop_batch(ctx):
    import bem_b200 as bb
    parts = bb.c4_particles(seed=5, count=3, ntheta=19)
    parts[1] = dict(parts[1], ka=-1.0)   # rejected by the pipeline's argument check
    out = bb.batch_run(ctx, parts, raise_on_error=False)
    assert [o[1]["status"] for o in out] == [0, 1, 0]
    assert np.all(out[0][0][0, 0] > 0) and np.all(out[2][0][0, 0] > 0)
    with pytest.raises(bb.BemError):
        bb.batch_run(ctx, parts)
