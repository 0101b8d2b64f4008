"""ctypes view of oracle/_ref/libref_host.so: the reference's own host C++
(mesh.cpp, rwg.cpp, rhs.cpp, orient.cpp, graglia.h) built by oracle/Makefile.

TEST INFRASTRUCTURE ONLY.  ``available()`` is False when the library has not
been built (for instance on a machine without the reference sources)."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_ref", "libref_host.so")
_lib = None


def available() -> bool:
    return os.path.exists(_LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(_LIB_PATH)
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def make_mesh(kind: str, param: float, ref: int):
    """kind 'ico' -> icosphere(radius=param, ref); 'hex' -> hex_prism(AR=param, ref).
    Returns (verts, tris, rwg-dict) in the reference's own RWG order."""
    L = lib()
    nv, nt, nr = C.c_int(), C.c_int(), C.c_int()
    L.ref_make_mesh(0 if kind == "ico" else 1, C.c_double(param), ref,
                    C.byref(nv), C.byref(nt), C.byref(nr))
    return _fetch(nv.value, nt.value, nr.value)


def load_obj(path):
    """The reference's load_obj on an existing file -> (verts, tris).  Its
    counts of removed degenerate triangles and of non-manifold edges go to
    stderr (mesh.cpp:220-245)."""
    L = lib()
    nv, nt = C.c_int(), C.c_int()
    L.ref_load_obj.argtypes = [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.ref_load_obj(str(path).encode(), C.byref(nv), C.byref(nt))
    verts = np.zeros((nv.value, 3))
    tris = np.zeros((nt.value, 3), dtype=np.int32)
    L.ref_get_mesh(_p(verts), _p(tris))
    return verts, tris


def mesh_utils(verts, tris):
    """The reference's mesh_volume, mesh_dmax and normalize_mesh on (verts,
    tris) -> (volume, dmax, a_eq, normalised verts)."""
    L = lib()
    v = np.ascontiguousarray(verts, dtype=np.float64)
    t = np.ascontiguousarray(tris, dtype=np.int32)
    L.ref_set_mesh(_p(v), len(v), _p(t), len(t))
    for f in (L.ref_mesh_volume, L.ref_mesh_dmax, L.ref_normalize_mesh):
        f.restype = C.c_double
    vol, dmax = L.ref_mesh_volume(), L.ref_mesh_dmax()
    a_eq = L.ref_normalize_mesh()
    vn = np.zeros_like(v)
    tn = np.zeros_like(t)
    L.ref_get_mesh(_p(vn), _p(tn))
    return vol, dmax, a_eq, vn


def rwg_of(verts, tris):
    """The reference's build_rwg on (verts, tris) -> the rwg dict of make_mesh."""
    L = lib()
    v = np.ascontiguousarray(verts, dtype=np.float64)
    t = np.ascontiguousarray(tris, dtype=np.int32)
    L.ref_set_mesh(_p(v), len(v), _p(t), len(t))
    nr = L.ref_build_rwg()
    return _fetch(len(v), len(t), nr)[2]


def singular_corrections(k, quad_order, N):
    """The reference's apply_singular_corrections (assembly.cu:208-321) on the
    mesh and RWG of the last make_mesh / rwg_of call, into a zero N x N L."""
    L = np.zeros((N, N), dtype=np.complex128)
    k = complex(k)
    lib().ref_singular_corrections(int(quad_order), C.c_double(k.real), C.c_double(k.imag), _p(L))
    return L


def subdivide_flat(verts, tris):
    """The reference's subdivide_flat (mesh.cpp:70-100) on (verts, tris) ->
    (verts, tris, rwg dict of the subdivided mesh)."""
    L = lib()
    v = np.ascontiguousarray(verts, dtype=np.float64)
    t = np.ascontiguousarray(tris, dtype=np.int32)
    L.ref_set_mesh(_p(v), len(v), _p(t), len(t))
    nr = L.ref_subdivide_flat()
    nv, nt = C.c_int(), C.c_int()
    L.ref_mesh_counts.argtypes = [C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.ref_mesh_counts(C.byref(nv), C.byref(nt))
    return _fetch(nv.value, nt.value, nr)


def tri_quadrature(order):
    """The reference's tri_quadrature(order) -> (pts (n, 2), wts (n,))."""
    pts, wts = np.zeros(50), np.zeros(25)
    n = lib().ref_tri_quadrature(int(order), _p(pts), _p(wts))
    return pts[:2 * n].reshape(n, 2), wts[:n]


def write_json(path, M, theta, ka, n_re, n_im, refinements, orient, times):
    """The reference's write_json; M (4, 4, ntheta), theta in radians."""
    Mf = np.ascontiguousarray(M, dtype=np.float64).reshape(-1)
    th = np.ascontiguousarray(theta, dtype=np.float64)
    d = C.c_double
    lib().ref_write_json(str(path).encode(), _p(Mf), _p(th), len(th), d(ka), d(n_re), d(n_im), int(refinements),
                         int(orient[0]), int(orient[1]), int(orient[2]), *[d(x) for x in times])


def farfield_cpu(cJ, cM, k_ext, eta_ext, r_hats, quad_order=7):
    """compute_far_field_vec_batch_cpu on the mesh of the last make_mesh call:
    cJ, cM (N,) complex, r_hats (ndir, 3) -> Fv (ndir, 3) complex."""
    cJ = np.ascontiguousarray(cJ, dtype=np.complex128)
    cM = np.ascontiguousarray(cM, dtype=np.complex128)
    rh = np.ascontiguousarray(r_hats, dtype=np.float64)
    Fv = np.zeros((len(rh), 3), dtype=np.complex128)
    k = complex(k_ext)
    lib().ref_farfield_cpu(int(quad_order), _p(cJ), _p(cM), C.c_double(k.real), C.c_double(k.imag),
                           C.c_double(eta_ext), _p(rh), len(rh), _p(Fv))
    return Fv


def amplitude_to_mueller(S1, S2, S3, S4):
    """The reference's amplitude_to_mueller -> M (4, 4, ntheta)."""
    S = [np.ascontiguousarray(x, dtype=np.complex128) for x in (S1, S2, S3, S4)]
    M = np.zeros(16 * len(S[0]))
    lib().ref_amplitude_to_mueller(*[_p(x) for x in S], len(S[0]), _p(M))
    return M.reshape(4, 4, -1)


def _fetch(nv, nt, nr):
    L = lib()
    verts = np.zeros((nv, 3))
    tris = np.zeros((nt, 3), dtype=np.int32)
    L.ref_get_mesh(_p(verts), _p(tris))
    tp = np.zeros(nr, dtype=np.int32)
    tm = np.zeros(nr, dtype=np.int32)
    fp = np.zeros((nr, 3))
    fm = np.zeros((nr, 3))
    ln, ap, am = np.zeros(nr), np.zeros(nr), np.zeros(nr)
    L.ref_get_rwg(_p(tp), _p(tm), _p(fp), _p(fm), _p(ln), _p(ap), _p(am))
    rwg = {"N": nr, "tri_p": tp.astype(np.int64), "tri_m": tm.astype(np.int64),
           "free_p": fp, "free_m": fm, "length": ln, "area_p": ap, "area_m": am}
    return verts, tris.astype(np.int64), rwg


def rhs(k_ext: complex, eta_ext: float, E0, k_hat, quad_order: int, N: int):
    """compute_rhs_planewave on the mesh made by the last make_mesh call."""
    b = np.zeros(2 * N, dtype=np.complex128)
    E0 = np.ascontiguousarray(E0, dtype=np.float64)
    kh = np.ascontiguousarray(k_hat, dtype=np.float64)
    lib().ref_rhs(C.c_double(complex(k_ext).real), C.c_double(complex(k_ext).imag),
                  C.c_double(eta_ext), _p(E0), _p(kh), quad_order, _p(b))
    return b


def orientations(na, nb, ng, beta_sym=1, gamma_sym=1, gamma_mirror=False, sort=False):
    n = lib().ref_orientations(na, nb, ng, beta_sym, gamma_sym, int(gamma_mirror), int(sort))
    RT = np.zeros((n, 3, 3))
    w = np.zeros(n)
    lib().ref_get_orientations(_p(RT), _p(w))
    return RT, w


def graglia(r, v0, v1, v2, quad_order=7):
    """(P, V) = potential_integral_triangle and vector_potential_integral_triangle."""
    args = [np.ascontiguousarray(x, dtype=np.float64) for x in (r, v0, v1, v2)]
    P = np.zeros(1)
    V = np.zeros(3)
    lib().ref_graglia(*[_p(a) for a in args], quad_order, _p(P), _p(V))
    return float(P[0]), V
