"""Streamed orientations: the per-orientation Mueller stream, adaptive
orientation stopping (main.cpp:477-636 on the dense path) and the bem_cuda
command line with its JSON and .per_orient outputs."""
import json
import os
import struct
import subprocess

import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(REPO, "bem-cpp_b200", "bin", "bem_cuda")


@pytest.fixture(scope="module")
def ctx():
    import bem_b200 as bb
    c = bb.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def sphere():
    import bem_b200 as bb
    return bb.icosphere(1.0, 1)


def test_per_orient_stream_sums_to_the_average(ctx, sphere):
    import bem_b200 as bb
    v, t = sphere
    ka = 1.2
    M, info = bb.dense_run(ctx, v, t, ka, 1.33, orient=(4, 3, 2), ntheta=31, per_orient=True)
    Mo, wo = info["per_orient_mueller"], info["per_orient_weight"]
    assert info["n_computed"] == info["n_orient"] == len(wo) == 24
    # M_avg = sum_o w_o M_o / |k|^2 (main.cpp:844-845)
    assert rel(np.einsum("o,oijt->ijt", wo, Mo) / ka ** 2, M) < 1e-13
    _, w_ref = bb.generate_orientations(4, 3, 2, sort_nearest=True)
    assert np.allclose(wo, w_ref, rtol=0, atol=0)


def _csca(M, w_sum):
    nt = M.shape[-1]
    th = np.pi * np.arange(nt) / (nt - 1)
    return float(np.sum(M[0, 0, 3:nt - 3] / w_sum * np.sin(th[3:nt - 3])))


def test_adaptive_stop_follows_the_reference_rule(ctx, sphere):
    import bem_b200 as bb
    v, t = sphere
    kw = dict(orient=(12, 10, 1), ntheta=19, per_orient=True)
    Mfull, ifull = bb.dense_run(ctx, v, t, 1.0, 1.31, **kw)
    M, info = bb.dense_run(ctx, v, t, 1.0, 1.31, orient_tol=0.05, **kw)
    n_tot, n_done = info["n_orient"], info["n_computed"]
    assert n_tot == 120
    # replay the rule on the per-orientation stream: checks every 20 from 40 on
    Mo, wo = ifull["per_orient_mueller"], ifull["per_orient_weight"]
    prev, ok, stop = None, 0, n_tot
    for done in range(20, n_tot + 1, 20):
        if done < 40:
            continue
        avg = np.einsum("o,oijt->ijt", wo[:done], Mo[:done])
        c = _csca(avg, wo[:done].sum())
        if prev is not None:
            ok = ok + 1 if abs(c - prev) / abs(prev) < 0.05 else 0
            if ok >= 2:
                stop = done
                break
        prev = c
    assert n_done == stop < n_tot
    expect = np.einsum("o,oijt->ijt", wo[:stop], Mo[:stop]) * (wo.sum() / wo[:stop].sum())
    assert rel(M, expect) < 1e-12
    assert rel(M, Mfull) < 0.05
    # a tolerance nothing meets solves every orientation: the plain average
    M2, i2 = bb.dense_run(ctx, v, t, 1.0, 1.31, orient_tol=1e-300, **kw)
    assert i2["n_computed"] == n_tot
    assert rel(M2, Mfull) < 1e-13


def test_cli_json_and_per_orient_file(ctx, sphere, tmp_path):
    import bem_b200 as bb
    if not os.path.exists(CLI):
        pytest.skip("bem_cuda not built")
    out = tmp_path / "run.json"
    cmd = [CLI, "--ka", "1.0", "--ref", "1", "--ri", "1.31", "0.0", "--orient", "12", "10", "1",
           "--ntheta", "19", "--orient-tol", "0.05", "--out", str(out)]
    subprocess.run(cmd, check=True, capture_output=True, text=True, timeout=300)
    d = json.loads(out.read_text())
    v, t = sphere
    M, info = bb.dense_run(ctx, v, t, 1.0, 1.31, orient=(12, 10, 1), ntheta=19, orient_tol=0.05,
                           per_orient=True)
    assert d["ntheta"] == 19 and d["orient"] == [12, 10, 1]
    assert rel(np.array(d["mueller"]), M) < 1e-7        # %.8e in the file
    raw = (tmp_path / "run.json.per_orient").read_bytes()
    n, nt, na, nb = struct.unpack("4i", raw[:16])
    assert (n, nt, na, nb) == (info["n_computed"], 19, 12, 10)
    w = np.frombuffer(raw[16:16 + 8 * n])
    Mo = np.frombuffer(raw[16 + 8 * n:]).reshape(n, 4, 4, nt)
    assert np.array_equal(w, info["per_orient_weight"])
    assert rel(Mo, info["per_orient_mueller"]) < 1e-15
