"""The reference's C++ call surface run on the GPU.

tests/compat/dense_branch.cpp makes the calls of the reference's dense
branch (main.cpp:660-854) through include/bem/*.h and libbem_compat.so --
assemble_pmchwt, lu_factorize_cuda + lu_solve_cuda, lu_solve_full,
compute_rhs_planewave, compute_far_field, FFCacheGPU +
compute_farfield_batch_cuda, amplitude_to_mueller, write_json (solver.h:11-22,
pmchwt.h:12-18, farfield.h:9-71, output.h) -- at the C1 size (icosphere
refinement 2, 2N = 960, ka = 1, m = 1.3116, the validate.py case), and
writes what each call returned.  The results are checked against the oracle
(the same RWG order) and against the reference's own outputs in
tests/golden/c1_single.npz (its Python RWG order, matched by triangle pair
and sign), and a singular matrix must come back as LAPACK's info."""
import json
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import load_golden, rel
from oracle import bem_oracle as bo

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(REPO, "bem-cpp_b200", "lib")
ORIENT = (3, 2, 1)
NTHETA = 181


def _build(tmp_path):
    cxx = shutil.which("g++")
    assert cxx, "no C++ compiler"
    exe = tmp_path / "dense_branch"
    cmd = [cxx, "-O1", "-std=c++17", "-Wall", "-Werror",
           "-I" + os.path.join(REPO, "include", "bem"), "-I" + os.path.join(REPO, "include"),
           "-o", str(exe), os.path.join(REPO, "tests", "compat", "dense_branch.cpp"),
           "-L" + LIB, "-Wl,-rpath," + LIB, "-lbem_compat", "-lbemdense"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    return exe


def _read(path, shape):
    return np.fromfile(path, dtype=np.complex128).reshape(shape)


def _mueller(path):
    with open(path) as f:
        d = json.load(f)
    return np.asarray(d["mueller"], dtype=np.float64), d


def _perm(rwg_cpp, rwg_py):
    """C++-order RWG i is Python-order RWG perm[i] times sign[i] (the same
    interior edge: the same pair of triangles, '+' and '-' maybe swapped)."""
    key = {}
    for j, (p, m) in enumerate(zip(rwg_py["tri_p"], rwg_py["tri_m"])):
        key[(int(p), int(m))] = (j, 1.0)
        key[(int(m), int(p))] = (j, -1.0)
    perm, sign = zip(*(key[(int(p), int(m))] for p, m in zip(rwg_cpp["tri_p"], rwg_cpp["tri_m"])))
    return np.array(perm), np.array(sign)


@pytest.fixture(scope="module")
def run(tmp_path_factory):
    tmp = tmp_path_factory.mktemp("compat")
    exe = _build(tmp)
    out = tmp / "out"
    out.mkdir()
    args = [str(exe), str(out), "2", "1.0", "1.3116", "0", *map(str, ORIENT), str(NTHETA)]
    r = subprocess.run(args, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (r.returncode, r.stdout[-2000:], r.stderr[-2000:])
    return out


def test_assemble_pmchwt_through_the_surface(run):
    import bem_b200 as bb
    v, t = bb.icosphere(1.0, 2)
    tt = t.astype(np.int64)
    rwg = bo.build_rwg(v, tt, "cpp")
    n = 2 * rwg["N"]
    Z = _read(run / "Z.bin", (n, n))
    Zo = bo.assemble_pmchwt(rwg, v, tt, 1.0, 1.3116, 1.0, 1.0 / 1.3116, 7)
    assert rel(Z, Zo) < 1e-12
    # the reference's own Z (bem_core, its RWG order): norm and diagonal
    gd = load_golden("c1_single.npz")
    perm, _ = _perm(rwg, {"tri_p": gd["rwg_tri_p"], "tri_m": gd["rwg_tri_m"]})
    assert abs(np.linalg.norm(Z) - gd["fro"]) / gd["fro"] < 1e-9
    full = np.concatenate([perm, perm + rwg["N"]])
    assert rel(np.diag(Z), gd["diag"][full]) < 1e-9


def test_lu_factorize_solve_and_solve_full_through_the_surface(run):
    import bem_b200 as bb
    v, t = bb.icosphere(1.0, 2)
    tt = t.astype(np.int64)
    rwg = bo.build_rwg(v, tt, "cpp")
    N = rwg["N"]
    n = 2 * N
    Z = _read(run / "Z.bin", (n, n))
    B = _read(run / "B1.bin", (2, n)).T
    X1 = _read(run / "X1.bin", (2, n)).T
    Xf = _read(run / "Xfull1.bin", (2, n)).T
    ipiv = np.fromfile(run / "ipiv.bin", dtype=np.int32)
    from scipy.linalg import lu_factor, lu_solve
    lu, piv = lu_factor(Z)
    assert np.array_equal(ipiv, piv + 1)          # LAPACK's pivots, 1-based as the reference returns them
    Xr = lu_solve((lu, piv), B)
    assert rel(X1, Xr) < 1e-11 and rel(Xf, X1) < 1e-12
    assert np.linalg.norm(Z @ X1 - B) / np.linalg.norm(B) < 1e-12
    # against the reference's solution of its own Z (bem_core, RWG order and sign mapped)
    gd = load_golden("c1_single.npz")
    perm, sign = _perm(rwg, {"tri_p": gd["rwg_tri_p"], "tri_m": gd["rwg_tri_m"]})
    full = np.concatenate([perm, perm + N])
    s2 = np.concatenate([sign, sign])[:, None]
    assert rel(B, s2 * gd["B"][full]) < 1e-12
    assert rel(X1, s2 * gd["X"][full]) < 1e-7   # the reference's Z carries ~1e-10 distance-expansion noise
    # every orientation through lu_solve_full
    no = ORIENT[0] * ORIENT[1] * ORIENT[2]
    Xo = _read(run / "Xo.bin", (2 * no, n)).T
    RT, w = bb.generate_orientations(*ORIENT)
    Bo = bo.orientation_rhs(rwg, v, tt, [(R, 1.0) for R in RT], 1.0, 1.0, 7)
    assert rel(Xo, lu_solve((lu, piv), Bo)) < 1e-11


def test_far_field_and_json_through_the_surface(run):
    import bem_b200 as bb
    v, t = bb.icosphere(1.0, 2)
    gd = load_golden("c1_single.npz")
    M1, d1 = _mueller(run / "single.json")
    assert M1.shape == (4, 4, NTHETA)
    # write_json prints the Mueller elements with 9 significant digits
    assert rel(M1, gd["mueller"]) < 1e-7
    assert np.allclose(d1["theta"], np.degrees(gd["theta"]), atol=1e-4)
    Mo, _ = _mueller(run / "orient.json")
    ctx = bb.Context(0)
    try:
        Mp, _ = bb.dense_run(ctx, v, t, 1.0, 1.3116, orient=ORIENT, ntheta=NTHETA)
    finally:
        ctx.close()
    assert rel(Mo, Mp) < 1e-7
    # compute_far_field of the single orientation's x column against the oracle
    tt = t.astype(np.int64)
    rwg = bo.build_rwg(v, tt, "cpp")
    N = rwg["N"]
    X1 = _read(run / "X1.bin", (2, 2 * N))
    F = _read(run / "Fsingle.bin", (2, NTHETA))
    cache = bo.FarFieldCache(rwg, v, tt, 7)
    th = np.linspace(0.0, np.pi, NTHETA)
    rh = np.stack([np.sin(th), np.zeros_like(th), np.cos(th)], axis=1)
    Fv = bo.far_field_vec(cache, X1[0, :N], X1[0, N:], 1.0, 1.0, rh)
    e_th = np.stack([np.cos(th), np.zeros_like(th), -np.sin(th)], axis=1)
    e_ph = np.tile([0.0, 1.0, 0.0], (NTHETA, 1))
    # (for this sphere and x polarisation F_phi vanishes in the phi = 0 plane
    # up to rounding: compare on the scale of F_theta)
    Ft, Fp = np.sum(Fv * e_th, axis=1), np.sum(Fv * e_ph, axis=1)
    assert rel(F[0], Ft) < 1e-12
    assert np.abs(F[1] - Fp).max() < 1e-12 * np.abs(Ft).max()


def test_singular_matrix_reports_lapack_info(run):
    import bem_b200 as bb
    v, t = bb.icosphere(1.0, 2)
    N = bb.build_rwg(v, t)["N"]
    info, full = (int(x) for x in open(run / "singular.txt").read().split())
    assert info == N + 1      # the zeroed column N is the first zero pivot (1-based)
    assert full == N + 1      # lu_solve_full returns the same info, as the reference's does


def test_geometry_cache_of_the_surface(tmp_path):
    # compute_rhs_planewave and FFCacheGPU::upload take host meshes call by
    # call and share device geometries kept by content: six distinct meshes
    # (more than the four unused geometries kept), the first again, the
    # first with one vertex moved, and far-field uploads of two meshes in
    # turn must each give what a fresh geometry of that mesh gives
    import bem_b200 as bb
    cxx = shutil.which("g++")
    exe = tmp_path / "geom_cache"
    r = subprocess.run([cxx, "-O1", "-std=c++17", "-Wall", "-Werror",
                        "-I" + os.path.join(REPO, "include", "bem"), "-I" + os.path.join(REPO, "include"),
                        "-o", str(exe), os.path.join(REPO, "tests", "compat", "geom_cache.cpp"),
                        "-L" + LIB, "-Wl,-rpath," + LIB, "-lbem_compat", "-lbemdense"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    out = tmp_path / "out"
    out.mkdir()
    r = subprocess.run([str(exe), str(out)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (r.stdout[-1500:], r.stderr[-1500:])
    meshes = [bb.icosphere(1.0, 1), bb.hex_prism(1.3, 1), bb.icosphere(0.7, 1), bb.hex_prism(0.8, 1),
              bb.icosphere(1.0, 2), bb.hex_prism(1.5, 2)]
    ctx = bb.Context(0)
    try:
        def fresh(v, t):
            g = bb.Geometry(ctx, v, t, 7)
            B = bb.rhs_planewave_dev(g, 2.0, 1.0, np.eye(3)[None])[0].cpu().numpy()
            g.close()
            return B
        got = [np.fromfile(out / f"rhs{i}.bin", dtype=np.complex128) for i in range(len(meshes))]
        for (v, t), b in zip(meshes, got):
            assert rel(b, fresh(v, t)) < 1e-14
        again = np.fromfile(out / "rhs0_again.bin", dtype=np.complex128)
        assert np.array_equal(again, got[0])
        v0, t0 = meshes[0]
        vm = np.array(v0, dtype=np.float64).copy()
        vm[0] *= 1.05
        moved = np.fromfile(out / "rhs0_moved.bin", dtype=np.complex128)
        assert rel(moved, got[0]) > 1e-6
        assert rel(moved, fresh(vm, t0)) < 1e-14
    finally:
        ctx.close()
    ff0, ff1, ff0b = (np.fromfile(out / f, dtype=np.complex128) for f in ("ff0.bin", "ff1.bin", "ff0_again.bin"))
    assert np.array_equal(ff0, ff0b) and np.all(np.isfinite(ff0))
    assert rel(ff1, ff0) > 1e-3
