"""C ABI checks that need no GPU: the library loads, exports every entry point
of include/bem_dense.h, and its host-side geometry matches the reference's own
C++ (oracle/_ref) and the oracle."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import REPO, rel
from oracle import bem_oracle as bo
from oracle import ref_host


def test_library_exports_every_declared_entry_point():
    import bem_b200 as bb
    from bem_b200 import _lib
    hdr = open(os.path.join(REPO, "include", "bem_dense.h")).read()
    declared = set(re.findall(r"^\s*(?:int|double|const char\*|int64_t)\s+(bem_\w+)\(", hdr, re.M))
    assert declared, "no declarations parsed"
    assert declared == set(_lib.SIGNATURES), declared ^ set(_lib.SIGNATURES)
    L = bb.lib()
    missing = [n for n in declared if not hasattr(L, n)]
    assert not missing, missing


def test_no_gpu_context_fails_cleanly():
    import torch
    import bem_b200 as bb
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    s = bb.lib().bem_ctx_create(0, C.byref(h))
    assert s == 7  # BEM_ERR_NODEVICE, no exit()


@pytest.mark.parametrize("ref", [0, 1, 2, 3])
def test_icosphere_and_rwg_match_reference_cpp(ref):
    import bem_b200 as bb
    if not ref_host.available():
        pytest.skip("oracle/_ref not built")
    v, t = bb.icosphere(1.0, ref)
    vr, tr, rr = ref_host.make_mesh("ico", 1.0, ref)
    assert np.array_equal(t, tr) and np.abs(v - vr).max() == 0.0
    r = bb.build_rwg(v, t)
    for k in ("tri_p", "tri_m"):
        assert np.array_equal(r[k], rr[k])
    for k in ("free_p", "free_m", "length", "area_p", "area_m"):
        assert np.abs(r[k] - rr[k]).max() == 0.0, k


@pytest.mark.parametrize("ar,ref", [(1.4286, 2), (0.7, 1), (2.0, 3)])
def test_hex_prism_matches_reference_cpp(ar, ref):
    import bem_b200 as bb
    if not ref_host.available():
        pytest.skip("oracle/_ref not built")
    v, t = bb.hex_prism(ar, ref)
    vr, tr, rr = ref_host.make_mesh("hex", ar, ref)
    assert np.array_equal(t, tr) and np.abs(v - vr).max() == 0.0
    assert bb.build_rwg(v, t)["N"] == rr["N"]


def test_hex_sizes_are_the_reference_mesher_sizes():
    # hex_prism starts at 24 triangles: ref 2 -> 2N = 1152, ref 3 -> 2N = 4608
    import bem_b200 as bb
    assert 2 * bb.build_rwg(*bb.hex_prism(1.4286, 2))["N"] == 1152
    assert 2 * bb.build_rwg(*bb.hex_prism(1.4286, 3))["N"] == 4608
    assert 2 * bb.build_rwg(*bb.icosphere(1.0, 5))["N"] == 61440


def test_subdivide_volume_dmax_normalize():
    import bem_b200 as bb
    v, t = bb.hex_prism(1.0, 0)
    v2, t2 = bb.subdivide_flat(v, t)
    vo, to = bo.subdivide_flat(v, t.astype(np.int64))
    assert np.array_equal(t2, to) and np.abs(v2 - vo).max() == 0.0
    assert abs(bb.mesh_volume(v, t) - 4 * np.pi / 3) < 1e-12
    vs, a = bb.normalize_mesh(3.0 * v, t)
    assert abs(a - 3.0) < 1e-12 and abs(bb.mesh_volume(vs, t) - 4 * np.pi / 3) < 1e-12
    ext = v.max(0) - v.min(0)
    assert abs(bb.mesh_dmax(v) - np.linalg.norm(ext)) < 1e-15


def test_load_obj_removes_degenerates(tmp_path):
    import bem_b200 as bb
    v, t = bb.icosphere(1.0, 1)
    p = tmp_path / "m.obj"
    with open(p, "w") as f:
        for x in v:
            f.write(f"v {x[0]:.17g} {x[1]:.17g} {x[2]:.17g}\n")
        for tri in t:
            f.write(f"f {tri[0]+1}/1/1 {tri[1]+1}/2/2 {tri[2]+1}/3/3\n")
        f.write("f 1 1 2\n")  # repeated vertex -> removed
    v2, t2, nd, nm = bb.load_obj(p)
    assert nd == 1 and nm == 0 and np.array_equal(t2, t)
    assert np.abs(v2 - v).max() < 1e-15


def test_load_obj_matches_the_reference(tmp_path, capfd):
    # quads (fan-triangulated), a repeated-vertex face, a zero-area face of
    # three collinear vertices and a fin: a third triangle on an existing edge
    import re
    import bem_b200 as bb
    if not ref_host.available():
        pytest.skip("reference host library not built")
    v, t = bb.hex_prism(1.0, 0)
    extra = np.array([[0.0, 0.0, 5.0], [1.0, 1.0, 5.0], [2.0, 2.0, 5.0], [0.3, 0.2, 3.0]])
    nv0 = len(v)
    p = tmp_path / "m.obj"
    with open(p, "w") as f:
        f.write("# test mesh\n")
        for x in np.vstack([v, extra]):
            f.write(f"v {x[0]:.17g} {x[1]:.17g} {x[2]:.17g}\n")
        tl = [list(x) for x in t]
        # the first two triangles written as one quad when they share an edge
        a, b = tl[0], tl[1]
        shared = [x for x in a if x in b]
        if len(shared) == 2:
            (oa,), (ob,) = [x for x in a if x not in shared], [x for x in b if x not in shared]
            i = a.index(oa)
            quad = [a[i], a[(i + 1) % 3], ob, a[(i + 2) % 3]]
            f.write("f " + " ".join(f"{q + 1}/{q + 1}" for q in quad) + "\n")
            tl = tl[2:]
        for tri in tl:
            f.write("f " + " ".join(str(q + 1) for q in tri) + "\n")
        f.write(f"f {nv0 + 1} {nv0 + 1} {nv0 + 2}\n")            # repeated vertex
        f.write(f"f {nv0 + 1} {nv0 + 2} {nv0 + 3}\n")            # collinear: zero area
        e0, e1 = t[2][0], t[2][1]
        f.write(f"f {e0 + 1} {e1 + 1} {nv0 + 4}\n")              # fin on an existing edge
    capfd.readouterr()
    vr, tr = ref_host.load_obj(p)
    err = capfd.readouterr().err
    nd_ref = int(re.search(r"removed (\d+) degenerate", err).group(1))
    nm_ref = int(re.search(r"(\d+) non-manifold edges", err).group(1))
    v2, t2, nd, nm = bb.load_obj(p)
    assert np.array_equal(v2, vr) and np.array_equal(t2, tr)
    assert (nd, nm) == (nd_ref, nm_ref) == (2, 1)


@pytest.mark.parametrize("case", ["bumpy", "hex", "flat"])
def test_mesh_utilities_match_the_reference(case):
    # mesh_volume, mesh_dmax and normalize_mesh (with its bounding-sphere
    # fallback for a zero-volume mesh) against the reference's own C++
    import bem_b200 as bb
    if not ref_host.available():
        pytest.skip("reference host library not built")
    if case == "bumpy":
        v, t = bb.c5_mesh(3, refinements=2, rms=0.1)
    elif case == "hex":
        v, t = bb.hex_prism(0.6, 2)
        v = 3.7 * v + np.array([0.3, -1.1, 2.0])
    else:
        v = np.array([[0.0, 0.0, 0.0], [2.0, 0.0, 0.0], [0.0, 1.5, 0.0], [1.0, 1.0, 0.0]])
        t = np.array([[0, 1, 2], [1, 3, 2]])
    vol, dmax, a_eq, vn = ref_host.mesh_utils(v, t)
    assert bb.mesh_volume(v, t) == vol
    assert bb.mesh_dmax(v) == dmax
    v2, a2 = bb.normalize_mesh(v, t)
    assert a2 == a_eq and np.array_equal(v2, vn)


@pytest.mark.parametrize("case", ["open_square", "open_cap", "fin", "unused_vertex", "single"])
def test_rwg_edge_cases_match_the_reference(case):
    # only edges shared by exactly two triangles carry a basis function
    # (rwg.cpp:22): boundary edges of open surfaces and edges of three
    # triangles get none; unused vertices change nothing
    import bem_b200 as bb
    if not ref_host.available():
        pytest.skip("reference host library not built")
    if case == "open_square":
        v = np.array([[0.0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]])
        t = np.array([[0, 1, 2], [0, 2, 3]])
    elif case == "single":
        v = np.array([[0.0, 0, 0], [1, 0, 0], [0, 1, 0]])
        t = np.array([[0, 1, 2]])
    else:
        v, t = bb.icosphere(1.0, 1)
        if case == "open_cap":
            t = t[v[t].mean(axis=1)[:, 2] > -0.2]                 # the lower cap removed
        elif case == "fin":
            v = np.vstack([v, [[2.0, 2.0, 2.0]]])
            t = np.vstack([t, [[t[0][0], t[0][1], len(v) - 1]]])  # a third triangle on one edge
        else:
            v = np.vstack([v, [[5.0, 5.0, 5.0]]])
    r = ref_host.rwg_of(v, t)
    o = bb.build_rwg(v, t)
    assert o["N"] == r["N"]
    for k in ("tri_p", "tri_m", "free_p", "free_m", "length", "area_p", "area_m"):
        assert np.array_equal(o[k], r[k]), k


@pytest.mark.parametrize("order", [4, 7, 13])
def test_quadrature(order):
    import bem_b200 as bb
    p, w = bb.tri_quadrature(order)
    po, wo = bo.tri_quadrature(order)
    assert np.array_equal(p, po) and np.array_equal(w, wo)
    assert abs(w.sum() - 1.0) < 1e-12


@pytest.mark.parametrize("order", [4, 7, 13, 5])
def test_quadrature_matches_the_reference_cpp(order):
    # the C ABI rejects an unknown order; the drop-in C++ header falls back to
    # the 7-point rule as the reference does
    import bem_b200 as bb
    if not ref_host.available():
        pytest.skip("reference host library not built")
    pr, wr = ref_host.tri_quadrature(order)
    p, w = bb.tri_quadrature(order if order in (4, 7, 13) else 7)
    assert np.array_equal(p, pr) and np.array_equal(w, wr)


def test_write_json_matches_the_reference_bytewise(tmp_path):
    # the JSON of the drop-in write_json (libbem_compat.so) against the
    # reference's output.cpp for the same inputs: cluster_bem.py parses it
    import ctypes as C
    import os
    if not ref_host.available():
        pytest.skip("reference host library not built")
    so = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "bem-cpp_b200", "lib",
                      "libbem_compat.so")
    if not os.path.exists(so):
        pytest.skip("libbem_compat.so not built")
    rng = np.random.default_rng(4)
    nt = 19
    M = rng.standard_normal((4, 4, nt)) * 10.0 ** rng.uniform(-12, 3, (4, 4, nt))
    M[0, 0, 3] = 0.0
    M[1, 2, 5] = -0.0
    theta = np.linspace(0.0, np.pi, nt)
    args = dict(ka=5.123456789, n_re=1.3116, n_im=1e-4, refinements=3, orient=(8, 7, 2),
                times=(1.234, 20.5, 0.999, 23.456))
    ref_host.write_json(tmp_path / "ref.json", M, theta, **args)
    lib = C.CDLL(so)
    f = lib["_Z10write_jsonPKcPKdS2_idddiiiidddd"]      # write_json(const char*, const double*, ...)
    d = C.c_double
    Mf = np.ascontiguousarray(M.reshape(-1))
    f(str(tmp_path / "ours.json").encode(), Mf.ctypes.data_as(C.c_void_p), theta.ctypes.data_as(C.c_void_p), nt,
      d(args["ka"]), d(args["n_re"]), d(args["n_im"]), 3, 8, 7, 2, *[d(x) for x in args["times"]])
    assert (tmp_path / "ours.json").read_bytes() == (tmp_path / "ref.json").read_bytes()


def test_quadrature_rejects_unknown_order():
    import bem_b200 as bb
    with pytest.raises(bb.BemError):
        bb.tri_quadrature(5)


@pytest.mark.parametrize("args", [(8, 8, 1, 1, 1, False), (45, 31, 1, 1, 1, False),
                                  (4, 3, 2, 2, 6, True), (5, 4, 3, 1, 1, True),
                                  (1, 1, 1, 1, 1, False), (1, 7, 1, 1, 1, False), (6, 1, 5, 1, 1, False),
                                  (3, 5, 4, 2, 1, False), (2, 2, 6, 1, 3, True), (12, 9, 2, 2, 2, True)])
def test_orientations_match_reference_cpp(args):
    import bem_b200 as bb
    RT, w = bb.generate_orientations(*args)
    assert abs(w.sum() - 1.0) < 1e-12 or args[3] != 1 or args[5]
    if ref_host.available():
        RTr, wr = ref_host.orientations(*args)
        assert np.abs(RT - RTr).max() == 0.0 and np.abs(w - wr).max() == 0.0
        RTs, ws = bb.generate_orientations(*args, sort_nearest=True)
        RTrs, wrs = ref_host.orientations(*args, sort=True)
        assert np.abs(RTs - RTrs).max() == 0.0 and np.abs(ws - wrs).max() == 0.0


def test_gauss_legendre():
    import bem_b200 as bb
    x, w = bb.gauss_legendre(31)
    xo, wo = bo.gauss_legendre(31)
    assert np.abs(x - xo).max() == 0.0 and np.abs(w - wo).max() == 0.0


def test_amplitude_to_mueller_host():
    import bem_b200 as bb
    rng = np.random.default_rng(3)
    S = [rng.standard_normal(17) + 1j * rng.standard_normal(17) for _ in range(4)]
    assert rel(bb.amplitude_to_mueller(*S), bo.amplitude_to_mueller(*S)) < 1e-15


def _cli():
    import os
    p = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "bem-cpp_b200", "bin", "bem_cuda")
    if not os.path.exists(p):
        pytest.skip("bem_cuda not built")
    return p


def test_cli_accepts_every_reference_flag(tmp_path):
    # every option of the reference's main.cpp:94-181 with its arguments; the
    # missing OBJ file stops the run after parsing, before any device work
    import subprocess
    flags = ["--ka", "2", "--ri", "1.31", "0.001", "--ref", "2", "--orient", "4", "4", "1", "--ntheta", "19",
             "--quad", "7", "--out", str(tmp_path / "r.json"), "--solver", "dense", "--prec", "none",
             "--prec-r", "1.5", "--prec-bs", "64", "--prec-overlap", "1", "--digits", "3", "--gmres-tol", "1e-6",
             "--gmres-restart", "50", "--max-leaf", "64", "--shape", "hex", "--ar", "1.2", "--orient-tol", "1e-4",
             "--orient-sym", "1", "1", "--subdiv", "1", "--orient-range", "0", "4", "--single", "--gamma-mirror",
             "--orient-auto", "3", "--goi", "--obj", str(tmp_path / "missing.obj")]
    r = subprocess.run([_cli()] + flags, capture_output=True, text=True, timeout=60)
    assert "Unknown option" not in r.stderr, r.stderr
    assert r.returncode == 1 and "cannot open OBJ file" in r.stderr


def test_cli_help_and_argument_errors():
    import subprocess
    for h in ("--help", "-h"):
        r = subprocess.run([_cli(), h], capture_output=True, text=True, timeout=60)
        assert r.returncode == 0 and "--ka" in r.stdout and "--orient-range" in r.stdout
    r = subprocess.run([_cli(), "--ka", "1", "--no-such-flag"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "Unknown option: --no-such-flag" in r.stderr
    r = subprocess.run([_cli(), "--ref", "2"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "--ka must be positive" in r.stderr


@pytest.mark.parametrize("mesh", ["hex", "bumpy"])
def test_subdivide_flat_matches_the_reference(mesh):
    # midpoint subdivision without projection (mesh.cpp:70-100), then the RWG
    # of the refined mesh, against the reference's own C++
    import bem_b200 as bb
    if not ref_host.available():
        pytest.skip("reference host library not built")
    v, t = bb.hex_prism(0.9, 1) if mesh == "hex" else bb.c5_mesh(5, refinements=1, rms=0.1)
    vr, tr, rr = ref_host.subdivide_flat(v, t)
    v2, t2 = bb.subdivide_flat(v, t)
    assert np.array_equal(v2, vr) and np.array_equal(t2, tr)
    o = bb.build_rwg(v2, t2)
    for k in ("tri_p", "tri_m", "free_p", "free_m", "length", "area_p", "area_m"):
        assert np.array_equal(o[k], rr[k]), k
