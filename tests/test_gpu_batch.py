"""Batched particles (bem_batch_run): the seeded hex-prism workload, each
particle identical to its own bem_dense_run, one against the oracle, and a
failing particle that does not stop the batch."""
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
    parts = bb.c4_particles(seed=3, count=4, ntheta=37)
    out = bb.batch_run(ctx, parts)
    assert len(out) == 4
    for p, (M, info) in zip(parts, out):
        assert info["status"] == 0
        assert info["N"] in (576, 2304) and info["n_orient"] == 16
        kw = {k: v for k, v in p.items() if k != "meta"}
        M1, _ = bb.dense_run(ctx, **kw)
        assert np.array_equal(M, M1)
        assert np.all(np.isfinite(M)) and np.all(M[0, 0] > 0)


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
