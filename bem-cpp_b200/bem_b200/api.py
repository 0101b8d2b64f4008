"""Python host layer over libbemdense (the C ABI in include/bem_dense.h).

Function names and argument meanings mirror the reference's CPU interface for
the dense path (python/bem_core.py: icosphere, build_rwg, tri_quadrature,
assemble_pmchwt, compute_rhs_planewave, compute_mueller_matrix,
orientation_average_mueller_batched, amplitude_to_mueller) and its C++ one
(solver.h: lu_factorize_cuda / lu_solve_cuda / lu_solve_full).  Every numeric
step runs in the CUDA library; device buffers are torch tensors, used only as
memory and streams.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from ._lib import (ASM_GSMOOTH_EXACT, PRECOND_BLOCK_DIAG, PRECOND_DIAG, PRECOND_LU,  # noqa: F401
                   PRECOND_NONE, PREC_FP32_REFINE, PREC_FP64, SOLVER_GMRES_AEXT, SOLVER_LU, BemError,
                   GmresStats, Problem, Result, SolveStats, check, lib)


def _ptr(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


def _dptr(t):
    return C.c_void_p(t.data_ptr())


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


# ------------------------------------------------------------------ context
class Context:
    """A libbemdense context on one GPU; kernels run on torch's current stream
    of that device at construction time unless ``stream`` is given."""

    def __init__(self, device: int = 0, stream=None):
        import torch
        self.device = device
        h = C.c_void_p()
        check(lib().bem_ctx_create(device, C.byref(h)))
        self.h = h
        if stream is None:
            stream = torch.cuda.current_stream(device)
        self.stream = stream
        check(lib().bem_ctx_set_stream(self.h, C.c_void_p(stream.cuda_stream)), self.h)

    def check(self, status):
        check(status, self.h)

    def synchronize(self):
        self.check(lib().bem_ctx_synchronize(self.h))

    @property
    def launches(self) -> int:
        return int(lib().bem_ctx_launch_count(self.h))

    PROF_CLASSES = ("lu_update", "solve_update", "residual", "panel", "assembly", "farfield", "verify", "trsm",
                    "interchanges", "panel_update")

    def profile(self, enable=True):
        self.check(lib().bem_ctx_profile(self.h, int(bool(enable))))

    def profile_read(self):
        """{class: (launches, device ms, algorithmic flops, algorithmic bytes)}."""
        out = {}
        for i, name in enumerate(self.PROF_CLASSES):
            n, ms, fl, by = C.c_int64(), C.c_double(), C.c_double(), C.c_double()
            self.check(lib().bem_ctx_profile_read(self.h, i, C.byref(n), C.byref(ms),
                                                  C.byref(fl), C.byref(by)))
            out[name] = (n.value, ms.value, fl.value, by.value)
        return out

    def close(self):
        if self.h:
            lib().bem_ctx_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------- geometry
def _mesh_call(fn, *args):
    nv, nt = C.c_int(), C.c_int()
    check(fn(*args, C.byref(nv), C.byref(nt), None, None))
    v = np.zeros((nv.value, 3))
    t = np.zeros((nt.value, 3), dtype=np.int32)
    check(fn(*args, C.byref(nv), C.byref(nt), _ptr(v), _ptr(t)))
    return v, t


def icosphere(radius=1.0, refinements=2):
    """(verts, tris) -- mesh.cpp:11-68 / bem_core.py:24-61."""
    return _mesh_call(lib().bem_mesh_icosphere, C.c_double(radius), int(refinements))


def hex_prism(aspect_ratio=1.0, refinements=2):
    """(verts, tris) -- mesh.cpp:102-154."""
    return _mesh_call(lib().bem_mesh_hex_prism, C.c_double(aspect_ratio), int(refinements))


def subdivide_flat(verts, tris):
    v, t = _f64(verts), _i32(tris)
    nv, nt = C.c_int(), C.c_int()
    L = lib()
    check(L.bem_mesh_subdivide_flat(_ptr(v), len(v), _ptr(t), len(t), C.byref(nv), C.byref(nt),
                                    None, None))
    vo = np.zeros((nv.value, 3))
    to = np.zeros((nt.value, 3), dtype=np.int32)
    check(L.bem_mesh_subdivide_flat(_ptr(v), len(v), _ptr(t), len(t), C.byref(nv), C.byref(nt),
                                    _ptr(vo), _ptr(to)))
    return vo, to


def load_obj(path):
    """(verts, tris, n_degenerate_removed, n_nonmanifold_edges) -- mesh.cpp:156-250."""
    nv, nt, nd, nm = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    L = lib()
    p = str(path).encode()
    check(L.bem_mesh_load_obj(p, C.byref(nv), C.byref(nt), None, None, C.byref(nd), C.byref(nm)))
    v = np.zeros((nv.value, 3))
    t = np.zeros((nt.value, 3), dtype=np.int32)
    check(L.bem_mesh_load_obj(p, C.byref(nv), C.byref(nt), _ptr(v), _ptr(t), C.byref(nd),
                              C.byref(nm)))
    return v, t, nd.value, nm.value


def normalize_mesh(verts, tris):
    v, t = _f64(verts).copy(), _i32(tris)
    a = C.c_double()
    check(lib().bem_mesh_normalize(_ptr(v), len(v), _ptr(t), len(t), C.byref(a)))
    return v, a.value


def mesh_volume(verts, tris):
    v, t = _f64(verts), _i32(tris)
    return lib().bem_mesh_volume(_ptr(v), len(v), _ptr(t), len(t))


def mesh_dmax(verts):
    v = _f64(verts)
    return lib().bem_mesh_dmax(_ptr(v), len(v))


def build_rwg(verts, tris):
    """RWG dict like bem_core.build_rwg, in the C++ edge order (rwg.cpp:5-43)."""
    v, t = _f64(verts), _i32(tris)
    N = C.c_int()
    L = lib()
    check(L.bem_rwg_build(_ptr(v), len(v), _ptr(t), len(t), C.byref(N), *([None] * 7)))
    n = N.value
    tp, tm = np.zeros(n, np.int32), np.zeros(n, np.int32)
    fp, fm = np.zeros((n, 3)), np.zeros((n, 3))
    ln, ap, am = np.zeros(n), np.zeros(n), np.zeros(n)
    check(L.bem_rwg_build(_ptr(v), len(v), _ptr(t), len(t), C.byref(N), _ptr(tp), _ptr(tm),
                          _ptr(fp), _ptr(fm), _ptr(ln), _ptr(ap), _ptr(am)))
    return {"N": n, "tri_p": tp.astype(np.int64), "tri_m": tm.astype(np.int64),
            "free_p": fp, "free_m": fm, "length": ln, "area_p": ap, "area_m": am}


def tri_quadrature(order=7):
    n = C.c_int()
    L = lib()
    check(L.bem_tri_quadrature(int(order), C.byref(n), None, None))
    p = np.zeros((n.value, 2))
    w = np.zeros(n.value)
    check(L.bem_tri_quadrature(int(order), C.byref(n), _ptr(p), _ptr(w)))
    return p, w


def generate_orientations(n_alpha, n_beta, n_gamma, beta_sym=1, gamma_sym=1,
                          gamma_mirror=False, sort_nearest=False):
    """(RT (n,3,3), weights (n,)) -- orient.cpp:73-163."""
    n = C.c_int()
    L = lib()
    args = (int(n_alpha), int(n_beta), int(n_gamma), int(beta_sym), int(gamma_sym),
            int(bool(gamma_mirror)), int(bool(sort_nearest)))
    check(L.bem_orientations(*args, C.byref(n), None, None))
    RT = np.zeros((n.value, 3, 3))
    w = np.zeros(n.value)
    check(L.bem_orientations(*args, C.byref(n), _ptr(RT), _ptr(w)))
    return RT, w


def gauss_legendre(n):
    x, w = np.zeros(n), np.zeros(n)
    check(lib().bem_gauss_legendre(int(n), _ptr(x), _ptr(w)))
    return x, w


def physics(ka, m):
    """k_ext = ka, k_int = k_ext m, eta_ext = 1, eta_int = 1/|m| (main.cpp:192-196)."""
    m = complex(m)
    return complex(ka, 0.0), complex(ka, 0.0) * m, 1.0, 1.0 / abs(m)


class Geometry:
    """Device-resident mesh + RWG + quadrature data (bem_geom)."""

    def __init__(self, ctx: Context, verts, tris, quad_order=7):
        self.ctx = ctx
        self.verts = _f64(verts)
        self.tris = _i32(tris)
        h = C.c_void_p()
        N = C.c_int()
        ctx.check(lib().bem_geom_create(ctx.h, _ptr(self.verts), len(self.verts),
                                        _ptr(self.tris), len(self.tris), int(quad_order),
                                        C.byref(h), C.byref(N)))
        self.h = h
        self.N = N.value
        self.n = 2 * self.N
        self.quad_order = quad_order

    @classmethod
    def from_rwg(cls, ctx: Context, verts, tris, rwg, quad_order=7):
        """Geometry with an explicit RWG basis (dict of build_rwg arrays: tri_p,
        tri_m, free_p, free_m, length, area_p, area_m), e.g. the reference
        Python build_rwg's order (bem_core.py:397-421)."""
        self = cls.__new__(cls)
        self.ctx = ctx
        self.verts = _f64(verts)
        self.tris = _i32(tris)
        arr = {k: (_i32(rwg[k]) if k in ("tri_p", "tri_m") else _f64(rwg[k]))
               for k in ("tri_p", "tri_m", "free_p", "free_m", "length", "area_p", "area_m")}
        self._rwg = arr
        N = len(arr["tri_p"])
        h = C.c_void_p()
        ctx.check(lib().bem_geom_create_rwg(
            ctx.h, _ptr(self.verts), len(self.verts), _ptr(self.tris), len(self.tris), N,
            _ptr(arr["tri_p"]), _ptr(arr["tri_m"]), _ptr(arr["free_p"]), _ptr(arr["free_m"]),
            _ptr(arr["length"]), _ptr(arr["area_p"]), _ptr(arr["area_m"]), int(quad_order),
            C.byref(h)))
        self.h = h
        self.N = N
        self.n = 2 * N
        self.quad_order = quad_order
        return self

    def set_vertices(self, verts):
        """Moves the mesh vertices in place (same topology; bem_geom_set_vertices)."""
        v = _f64(verts)
        assert v.shape == self.verts.shape
        self.ctx.check(lib().bem_geom_set_vertices(self.ctx.h, self.h, _ptr(v)))
        self.verts = v

    def close(self):
        if self.h:
            lib().bem_geom_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _empty(shape, dtype, device):
    import torch
    return torch.empty(shape, dtype=dtype, device=f"cuda:{device}")


def assemble_pmchwt_dev(geom: Geometry, k_ext, k_int, eta_ext, eta_int, Z=None,
                        exact_gsmooth=False):
    """Device Z (torch complex128, row-major 2N x 2N) -- pmchwt.cu:6-56."""
    import torch
    n = geom.n
    if Z is None:
        Z = _empty((n, n), torch.complex128, geom.ctx.device)
    assert Z.dtype == torch.complex128 and Z.is_contiguous() and Z.shape[0] == n
    k_ext, k_int = complex(k_ext), complex(k_int)
    geom.ctx.check(lib().bem_assemble_pmchwt_dev(
        geom.ctx.h, geom.h, k_ext.real, k_ext.imag, k_int.real, k_int.imag, float(eta_ext),
        float(eta_int), ASM_GSMOOTH_EXACT if exact_gsmooth else 0, _dptr(Z), Z.stride(0)))
    return Z


def assemble_L_K_dev(geom: Geometry, k, exact_gsmooth=False):
    """Device (L, K) for one wavenumber -- assemble_L_K_cuda, assembly.h:11-13."""
    import torch
    N = geom.N
    Lm = _empty((N, N), torch.complex128, geom.ctx.device)
    Km = _empty((N, N), torch.complex128, geom.ctx.device)
    k = complex(k)
    geom.ctx.check(lib().bem_assemble_LK_dev(geom.ctx.h, geom.h, k.real, k.imag,
                                             ASM_GSMOOTH_EXACT if exact_gsmooth else 0,
                                             _dptr(Lm), _dptr(Km), N))
    return Lm, Km


# ---------------------------------------------------------------------- LU
def _as_cols(B, n, device):
    """Column-major n x nrhs device buffer as a torch (nrhs, n) tensor."""
    import torch
    if isinstance(B, np.ndarray):
        B = torch.from_numpy(np.ascontiguousarray(np.asarray(B, dtype=np.complex128).reshape(n, -1).T))
    B = B.to(device=f"cuda:{device}", dtype=torch.complex128)
    if B.dim() == 1:
        B = B.reshape(1, n)
    return B.contiguous()


class LU:
    """Device-resident factorisation of a row-major complex128 Z (torch tensor).

    precision PREC_FP64: Z is overwritten by its factors (P Z = L U).
    precision PREC_FP32_REFINE: Z is kept (the FP64 refinement residual uses it;
    keep the tensor alive) and complex64 factors are made alongside."""

    def __init__(self, ctx: Context, Z, precision=PREC_FP64):
        import torch
        assert Z.dtype == torch.complex128 and Z.dim() == 2 and Z.stride(1) == 1
        self.ctx = ctx
        self.Z = Z
        self.n = Z.shape[0]
        self.precision = precision
        h = C.c_void_p()
        info = C.c_int()
        ctx.check(lib().bem_lu_factor_dev(ctx.h, _dptr(Z), self.n, Z.stride(0), int(precision),
                                          C.byref(h), C.byref(info)))
        self.h = h
        self.info = info.value

    def solve(self, B, X=None, tol=0.0, max_iter=0, raise_noconv=True):
        """X = Z^-1 B.  B: torch (nrhs, n) complex128 on the device (column c of
        the column-major n x nrhs right-hand side is row c), or a numpy (n, nrhs)
        array.  Returns (X as torch (nrhs, n), stats dict)."""
        B = _as_cols(B, self.n, self.ctx.device)
        if X is None:
            X = torch_empty_like(B)
        st = SolveStats()
        s = lib().bem_lu_solve_dev(self.ctx.h, self.h, _dptr(B), self.n, _dptr(X), self.n,
                                   B.shape[0], float(tol), int(max_iter), C.byref(st))
        if s != 0 and not (s == 5 and not raise_noconv):
            self.ctx.check(s)
        return X, st.as_dict()

    def residual(self, B, X, method=1):
        """R = B - Z X in FP64 (method 0: FP64 GEMM, 1: int8 Ozaki digits).
        B, X: torch (nrhs, n) complex128 on the device.  Returns R like B."""
        import torch
        assert B.shape == X.shape and B.dtype == X.dtype == torch.complex128
        B = B.contiguous()
        X = X.contiguous()
        R = torch.empty_like(B)
        self.ctx.check(lib().bem_lu_residual_dev(self.ctx.h, self.h, _dptr(B), self.n, _dptr(X), self.n,
                                                 _dptr(R), self.n, B.shape[0], int(method)))
        return R

    def close(self):
        if self.h:
            lib().bem_lu_free(self.h)
            self.h = None
        self.Z = None  # drop the reference to the (possibly 60 GB) matrix

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def torch_empty_like(t):
    import torch
    return torch.empty_like(t)


def lu_factorize_cuda(ctx: Context, Z):
    """Host mirror of solver.h:11 -- returns (factors, ipiv (1-based), info);
    the factors are those of the row-major Z (P Z = L U)."""
    Zc = np.ascontiguousarray(Z, dtype=np.complex128).copy()
    n = Zc.shape[0]
    ipiv = np.zeros(n, dtype=np.int32)
    info = C.c_int()
    ctx.check(lib().bem_lu_factorize(ctx.h, _ptr(Zc), n, _ptr(ipiv), C.byref(info)))
    return Zc, ipiv, info.value


def lu_solve_cuda(ctx: Context, Z_lu, ipiv, B):
    """Host mirror of solver.h:16-17: B (n,) or (n, nrhs) -> X."""
    n = Z_lu.shape[0]
    Bf = np.asfortranarray(np.asarray(B, dtype=np.complex128).reshape(n, -1)).copy(order="F")
    Zl = np.ascontiguousarray(Z_lu, dtype=np.complex128)
    ip = _i32(ipiv)
    ctx.check(lib().bem_lu_solve(ctx.h, _ptr(Zl), _ptr(ip), n,
                                 C.c_void_p(Bf.ctypes.data), Bf.shape[1]))
    return Bf.reshape(np.shape(B)) if np.ndim(B) == 1 else Bf


def lu_solve_full(ctx: Context, Z, B, precision=PREC_FP64):
    """Host mirror of solver.h:21-22: returns (X, stats)."""
    Zc = np.ascontiguousarray(Z, dtype=np.complex128).copy()
    n = Zc.shape[0]
    Bf = np.asfortranarray(np.asarray(B, dtype=np.complex128).reshape(n, -1)).copy(order="F")
    st = SolveStats()
    ctx.check(lib().bem_lu_solve_full(ctx.h, _ptr(Zc), n, C.c_void_p(Bf.ctypes.data), Bf.shape[1],
                                      int(precision), C.byref(st)))
    return (Bf.reshape(np.shape(B)) if np.ndim(B) == 1 else Bf), st.as_dict()


# --------------------------------------------------------------- excitation
# ------------------------------------------------------------------- GMRES
def assemble_aext_dev(geom: Geometry, k_ext, eta_ext, Z=None, exact_gsmooth=False):
    """Device A_ext = [[eta L_ext, -K_ext], [K_ext, L_ext / eta]] (torch complex128,
    row-major 2N x 2N) -- the matrix of build_aext_preconditioner, bem_core.py:1071-1090."""
    import torch
    n = geom.n
    if Z is None:
        Z = _empty((n, n), torch.complex128, geom.ctx.device)
    assert Z.dtype == torch.complex128 and Z.is_contiguous() and Z.shape[0] == n
    k_ext = complex(k_ext)
    geom.ctx.check(lib().bem_assemble_aext_dev(
        geom.ctx.h, geom.h, k_ext.real, k_ext.imag, float(eta_ext),
        ASM_GSMOOTH_EXACT if exact_gsmooth else 0, _dptr(Z), Z.stride(0)))
    return Z


_PRECOND = {None: PRECOND_NONE, "none": PRECOND_NONE, "diag": PRECOND_DIAG,
            "block_diag": PRECOND_BLOCK_DIAG, "aext": PRECOND_LU, "lu": PRECOND_LU}


class Preconditioner:
    """bem_precond: kind None / 'diag' / 'block_diag' built from Z (torch
    complex128, kept alive here), or 'aext' / 'lu' from an LU object (the
    factorisation of A_ext; kept alive here)."""

    def __init__(self, ctx: Context, kind, Z=None, n=None, precision=PREC_FP64, lu=None):
        if kind not in _PRECOND:
            raise ValueError(f"unknown preconditioner {kind!r}")
        self.ctx, self.kind, self.Z, self.lu = ctx, kind, Z, lu
        self.n = n if n is not None else (Z.shape[0] if Z is not None else lu.n)
        h = C.c_void_p()
        ctx.check(lib().bem_precond_create(ctx.h, _PRECOND[kind], _dptr(Z) if Z is not None else None,
                                           self.n, Z.stride(0) if Z is not None else self.n,
                                           int(precision), lu.h if lu is not None else None,
                                           C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            lib().bem_precond_free(self.h)
            self.h = None
        if self.lu is not None and getattr(self, "_own_lu", False):
            self.lu.close()
        self.Z = self.lu = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def build_aext_preconditioner(geom: Geometry, k_ext, eta_ext, precision=PREC_FP64, keep_matrix=False):
    """build_aext_preconditioner (bem_core.py:1071-1090): A_ext assembled on the
    device and factored.  Returns (Z_ext_lu, Z_ext) like the reference, where
    Z_ext_lu is a Preconditioner of kind 'aext' and Z_ext the unfactored matrix
    when keep_matrix (an FP64 factorisation overwrites its input, so keeping it
    costs a copy), else None.  precision PREC_FP32_REFINE factors A_ext in FP32
    (applied once per step, no refinement)."""
    A = assemble_aext_dev(geom, k_ext, eta_ext)
    Z_ext = A.clone() if keep_matrix else None
    lu = LU(geom.ctx, A, precision)
    M = Preconditioner(geom.ctx, "aext", lu=lu)
    M._own_lu = True
    return M, Z_ext


def gmres(ctx: Context, Z, B, M=None, tol=1e-5, restart=20, maxiter=None):
    """GMRES(restart) for Z X = B on the device, all columns of B at once (the
    algorithm of scipy.sparse.linalg.gmres that the reference calls).  Z: torch
    complex128 (n, n) on the device.  B: numpy (n,) / (n, nrhs), or torch
    (nrhs, n) on the device.  M: a Preconditioner (None: identity).  maxiter:
    restart cycles (default 10 n, scipy's).  Returns (X in B's form, info dict:
    'iters' and 'info' per column as scipy's callback count and info, and the
    batch statistics)."""
    import torch
    n = Z.shape[0]
    as_numpy = isinstance(B, np.ndarray)
    one = as_numpy and B.ndim == 1
    Bt = _as_cols(B, n, ctx.device)
    nrhs = Bt.shape[0]
    X = torch.empty_like(Bt)
    own = M is None
    if own:
        M = Preconditioner(ctx, None, n=n)
    iters = np.zeros(nrhs, dtype=np.int32)
    info = np.zeros(nrhs, dtype=np.int32)
    st = GmresStats()
    try:
        ctx.check(lib().bem_gmres_solve_dev(
            ctx.h, _dptr(Z), n, Z.stride(0), M.h, _dptr(Bt), n, _dptr(X), n, nrhs, int(restart),
            float(tol), int(maxiter if maxiter is not None else 10 * n), _ptr(iters), _ptr(info),
            C.byref(st)))
    finally:
        if own:
            M.close()
    d = st.as_dict()
    d["iters"], d["info"] = iters, info
    if as_numpy:
        Xh = X.cpu().numpy().T
        return (Xh[:, 0] if one else Xh), d
    return X, d


def solve_gmres_aext(ctx: Context, Z, b, Z_ext_lu, tol=1e-5, maxiter=200):
    """solve_gmres_aext (bem_core.py:1093-1123): GMRES with the A_ext
    preconditioner, restart min(200, n).  Returns x in b's form."""
    x, _ = gmres(ctx, Z, b, Z_ext_lu, tol=tol, restart=min(200, Z.shape[0]), maxiter=maxiter)
    return x


def solve_gmres(ctx: Context, Z, b, tol=1e-4, maxiter=500, precond="block_diag", Z_ext_lu=None,
                precision=PREC_FP64):
    """solve_gmres (bem_core.py:1126-1183): precond 'aext' (needs Z_ext_lu),
    'block_diag' (LU of Z11 and Z22), 'diag' or None; restart 20 (scipy's
    default) except for 'aext'.  precision: of the block factorisations."""
    if precond == "aext":
        if Z_ext_lu is None:
            raise ValueError("precond='aext' requires Z_ext_lu from build_aext_preconditioner()")
        return solve_gmres_aext(ctx, Z, b, Z_ext_lu, tol=tol, maxiter=maxiter)
    M = Preconditioner(ctx, precond, Z=Z, precision=precision)
    try:
        x, _ = gmres(ctx, Z, b, M, tol=tol, restart=20, maxiter=maxiter)
    finally:
        M.close()
    return x


def rhs_planewave_dev(geom: Geometry, k_ext, eta_ext, RT, B=None):
    """Right-hand sides for orientations RT (n,3,3): torch (2n_orient, 2N) whose
    row 2o is par (E0 = RT x), 2o+1 perp (E0 = RT y), k_hat = RT z
    (rhs.cpp:6-64, main.cpp:739-751)."""
    import torch
    RT = _f64(RT).reshape(-1, 9)
    no = RT.shape[0]
    if B is None:
        B = _empty((2 * no, geom.n), torch.complex128, geom.ctx.device)
    k = complex(k_ext)
    geom.ctx.check(lib().bem_rhs_planewave_dev(geom.ctx.h, geom.h, k.real, k.imag, float(eta_ext),
                                               _ptr(RT), no, _dptr(B), B.stride(0)))
    return B


def compute_rhs_planewave(geom: Geometry, k_ext, eta_ext, E0=(1.0, 0.0, 0.0),
                          k_hat=(0.0, 0.0, 1.0)):
    """b = [<f,E_inc>; <f,H_inc>] (host, complex128[2N]) -- rhs.h:11-15."""
    b = np.zeros(geom.n, dtype=np.complex128)
    k = complex(k_ext)
    E0, k_hat = _f64(E0), _f64(k_hat)  # keep the contiguous copies alive
    geom.ctx.check(lib().bem_rhs_planewave(geom.ctx.h, geom.h, k.real, k.imag, float(eta_ext),
                                           _ptr(E0), _ptr(k_hat),
                                           C.c_void_p(b.ctypes.data)))
    return b


# ------------------------------------------------------- far field, Mueller
def compute_farfield_batch(geom: Geometry, coeffs_J, coeffs_M, r_hats, k_ext, eta_ext):
    """compute_farfield_batch_cuda (farfield.h:35-48): coeffs (n_calls, N) complex,
    r_hats (n_orient, ndir, 3); returns Fv (n_calls, ndir, 3) complex."""
    cJ = np.ascontiguousarray(coeffs_J, dtype=np.complex128)
    cM = np.ascontiguousarray(coeffs_M, dtype=np.complex128)
    rh = _f64(r_hats)
    n_calls = cJ.shape[0]
    no, nd = rh.shape[0], rh.shape[1]
    Fv = np.zeros((n_calls, nd, 3), dtype=np.complex128)
    k = complex(k_ext)
    geom.ctx.check(lib().bem_farfield_batch(geom.ctx.h, geom.h, C.c_void_p(cJ.ctypes.data),
                                            C.c_void_p(cM.ctypes.data), _ptr(rh), k.real, k.imag,
                                            float(eta_ext), n_calls, no, nd,
                                            C.c_void_p(Fv.ctypes.data)))
    return Fv


def _check_solutions(geom: Geometry, X, RT, w):
    """Checks the solution tensor and orientation arrays handed to the far-field
    entry points as raw pointers: X complex128 on the geometry's device with
    unit stride along a solution and one (par, perp) pair of rows per
    orientation; one weight per orientation.  Returns (RT as (n, 9), w)."""
    import torch
    RT = _f64(RT).reshape(-1, 9)
    w = _f64(w).reshape(-1)
    if not (isinstance(X, torch.Tensor) and X.dtype == torch.complex128 and X.is_cuda
            and X.device.index == geom.ctx.device and X.dim() == 2):
        raise ValueError("X must be a 2-D complex128 tensor on the geometry's device")
    if X.stride(1) != 1 or X.shape[1] < geom.n or X.stride(0) < geom.n:
        raise ValueError(f"X rows must be contiguous solutions of length {geom.n}")
    if X.shape[0] < 2 * RT.shape[0]:
        raise ValueError(f"X has {X.shape[0]} rows, {2 * RT.shape[0]} needed for {RT.shape[0]} orientations")
    if w.size != RT.shape[0]:
        raise ValueError(f"{w.size} weights for {RT.shape[0]} orientations")
    return RT, w


def mueller_from_solutions_dev(geom: Geometry, X, RT, w, k_ext, eta_ext, ntheta=181,
                               gamma_mirror=False, M_orient=None):
    """Orientation-weighted Mueller sum (4,4,ntheta) from device solutions X
    (torch (2 n_orient, 2N), rows (par, perp) per orientation)."""
    import torch
    RT, w = _check_solutions(geom, X, RT, w)
    if M_orient is not None and not (
            isinstance(M_orient, torch.Tensor) and M_orient.dtype == torch.float64 and M_orient.is_cuda
            and M_orient.device.index == geom.ctx.device and M_orient.is_contiguous()
            and M_orient.numel() >= RT.shape[0] * 16 * int(ntheta)):
        raise ValueError("M_orient must be a contiguous float64 device tensor of n_orient*16*ntheta elements")
    M = np.zeros((4, 4, ntheta))
    k = complex(k_ext)
    geom.ctx.check(lib().bem_farfield_mueller_dev(
        geom.ctx.h, geom.h, _dptr(X), X.stride(0), _ptr(RT), _ptr(w), RT.shape[0], k.real, k.imag,
        float(eta_ext), int(ntheta), int(bool(gamma_mirror)), _ptr(M),
        _dptr(M_orient) if M_orient is not None else None))
    return M


def amplitude_to_mueller(S1, S2, S3, S4):
    """Bohren & Huffman 3.16 (farfield.cu:464-508) -> (4, 4, ntheta)."""
    S = [np.ascontiguousarray(s, dtype=np.complex128) for s in (S1, S2, S3, S4)]
    nt = len(S[0])
    M = np.zeros((4, 4, nt))
    check(lib().bem_amplitude_to_mueller(*[C.c_void_p(s.ctypes.data) for s in S], nt, _ptr(M)))
    return M


# ------------------------------------------------------------ whole pipeline
def dense_run(ctx: Context, verts, tris, ka, m=1.3116, quad_order=7, single=False,
              orient=(8, 8, 1), orient_sym=(1, 1), gamma_mirror=False, orient_range=None,
              ntheta=181, precision=PREC_FP64, refine_tol=0.0, max_refine=0, exact_gsmooth=False,
              orient_tol=0.0, per_orient=False, solver="lu", gmres_tol=0.0, gmres_restart=0,
              gmres_maxiter=0):
    """The --solver dense pipeline (main.cpp:660-854) through bem_dense_run.
    Returns (mueller (4,4,ntheta), info dict).  orient_tol > 0: adaptive
    orientation stopping (main.cpp:477-636); per_orient=True adds the
    per-orientation Mueller matrices and weights of the solved orientations to
    info ("per_orient_mueller" (n,4,4,ntheta), "per_orient_weight" (n,)).
    solver "gmres_aext": GMRES with the A_ext LU preconditioner instead of
    the LU of Z (bem_core.py:1703-1709); info["gmres"] has its statistics."""
    p, _keep = _problem(verts, tris, ka, m, quad_order, single, orient, orient_sym, gamma_mirror,
                        orient_range, ntheta, precision, refine_tol, max_refine, exact_gsmooth, orient_tol,
                        solver, gmres_tol, gmres_restart, gmres_maxiter)
    M = np.zeros((4, 4, ntheta))
    r = Result(mueller=M.ctypes.data)
    po_M = po_w = None
    if per_orient:
        cnt = 1 if single else len(generate_orientations(orient[0], orient[1], orient[2], orient_sym[0],
                                                         orient_sym[1], gamma_mirror)[1])
        po_M = np.zeros((cnt, 4, 4, ntheta))
        po_w = np.zeros(cnt)
        r.per_orient_mueller = po_M.ctypes.data
        r.per_orient_weight = po_w.ctypes.data
    ctx.check(lib().bem_dense_run(ctx.h, C.byref(p), C.byref(r)))
    info = {"N": r.N, "n_orient": r.n_orient, "n_computed": r.n_computed,
            "t_assembly_s": r.t_assembly_s, "t_solve_s": r.t_solve_s, "t_farfield_s": r.t_farfield_s,
            "t_total_s": r.t_total_s, "t_setup_s": r.t_setup_s, "t_release_s": r.t_release_s,
            "stats": r.stats.as_dict(), "gmres": r.gmres.as_dict()}
    if per_orient:
        info["per_orient_mueller"] = po_M[:r.n_computed]
        info["per_orient_weight"] = po_w[:r.n_computed]
    return M, info


def _problem(verts, tris, ka, m=1.3116, quad_order=7, single=False, orient=(8, 8, 1),
             orient_sym=(1, 1), gamma_mirror=False, orient_range=None, ntheta=181,
             precision=PREC_FP64, refine_tol=0.0, max_refine=0, exact_gsmooth=False, orient_tol=0.0,
             solver="lu", gmres_tol=0.0, gmres_restart=0, gmres_maxiter=0):
    solvers = {"lu": SOLVER_LU, "gmres_aext": SOLVER_GMRES_AEXT}
    if solver not in solvers:
        raise ValueError(f"unknown solver {solver!r} (lu, gmres_aext)")
    v, t = _f64(verts), _i32(tris)
    m = complex(m)
    i0, i1 = orient_range if orient_range is not None else (-1, -1)
    p = Problem(verts=v.ctypes.data, nv=len(v), tris=t.ctypes.data, nt=len(t), ka=float(ka),
                m_re=m.real, m_im=m.imag, quad_order=int(quad_order), single=int(bool(single)),
                n_alpha=int(orient[0]), n_beta=int(orient[1]), n_gamma=int(orient[2]),
                beta_sym=int(orient_sym[0]), gamma_sym=int(orient_sym[1]),
                gamma_mirror=int(bool(gamma_mirror)), orient_i0=int(i0), orient_i1=int(i1),
                ntheta=int(ntheta), precision=int(precision), refine_tol=float(refine_tol),
                max_refine=int(max_refine), asm_flags=ASM_GSMOOTH_EXACT if exact_gsmooth else 0,
                orient_tol=float(orient_tol), solver=solvers[solver], gmres_tol=float(gmres_tol),
                gmres_restart=int(gmres_restart), gmres_maxiter=int(gmres_maxiter))
    return p, (v, t)


def batch_run(ctx: Context, particles, raise_on_error=True):
    """Many particles through bem_batch_run.  `particles`: list of dicts with
    the keyword arguments of dense_run (verts, tris, ka, m, orient, ...; a
    "meta" entry is ignored).
    Returns a list of (mueller (4,4,ntheta), info) with info["status"] per
    particle (0 = OK)."""
    n = len(particles)
    probs = (Problem * max(n, 1))()
    res = (Result * max(n, 1))()
    keep, outs = [], []
    for i, kw in enumerate(particles):
        p, arrays = _problem(**{k: v for k, v in kw.items() if k != "meta"})
        keep.append(arrays)
        probs[i] = p
        M = np.zeros((4, 4, p.ntheta))
        outs.append(M)
        res[i].mueller = M.ctypes.data
    st = (C.c_int * max(n, 1))()
    s = lib().bem_batch_run(ctx.h, probs, n, res, st)
    if s != 0 and raise_on_error:
        ctx.check(s)
    out = []
    for i in range(n):
        r = res[i]
        out.append((outs[i], {"status": st[i], "N": r.N, "n_orient": r.n_orient,
                              "t_assembly_s": r.t_assembly_s, "t_solve_s": r.t_solve_s,
                              "t_farfield_s": r.t_farfield_s, "t_total_s": r.t_total_s,
                              "stats": r.stats.as_dict()}))
    return out


def adjoint_grad(ctx: Context, verts, tris, ka, m, target, wt=None, **kw):
    """Adjoint gradient of sum_t wt_t (M11(theta_t) - target_t)^2 with respect to
    (Re m, Im m).  `target` has one value per scattering angle (ntheta = len).
    Returns (loss, grad (2,), mueller (4, 4, ntheta))."""
    target = np.ascontiguousarray(target, dtype=np.float64)
    nt = len(target)
    p, keep = _problem(verts, tris, ka, m, ntheta=nt, **kw)
    wtv = None if wt is None else np.ascontiguousarray(wt, dtype=np.float64)
    loss = C.c_double()
    grad = np.zeros(2)
    M = np.zeros((4, 4, nt))
    ctx.check(lib().bem_adjoint_grad(ctx.h, C.byref(p), target.ctypes.data,
                                     None if wtv is None else wtv.ctypes.data, C.byref(loss),
                                     grad.ctypes.data, M.ctypes.data))
    return loss.value, grad, M


def adjoint_grad_vertices(ctx: Context, verts, tris, ka, m, target, wt=None, **kw):
    """Gradient of sum_t wt_t (M11(theta_t) - target_t)^2 with respect to the
    vertex coordinates.  Returns (loss, grad (nv, 3), mueller (4, 4, ntheta))."""
    target = np.ascontiguousarray(target, dtype=np.float64)
    nt = len(target)
    p, keep = _problem(verts, tris, ka, m, ntheta=nt, **kw)
    wtv = None if wt is None else np.ascontiguousarray(wt, dtype=np.float64)
    loss = C.c_double()
    grad = np.zeros((len(keep[0]), 3))
    M = np.zeros((4, 4, nt))
    ctx.check(lib().bem_adjoint_grad_vertices(ctx.h, C.byref(p), target.ctypes.data,
                                              None if wtv is None else wtv.ctypes.data, C.byref(loss),
                                              grad.ctypes.data, M.ctypes.data))
    return loss.value, grad, M


def _misfit_function():
    import torch

    class MuellerMisfit(torch.autograd.Function):
        """loss = sum_t wt_t (M11(theta_t) - target_t)^2 of the orientation-
        averaged Mueller matrix; the gradients come from the adjoint entry
        points (bem_adjoint_grad_vertices for the vertices, only when they
        require a gradient, and bem_adjoint_grad for m), computed together
        with the loss in the forward pass."""

        @staticmethod
        def forward(fctx, verts, m_re, m_im, bctx, tris, ka, target, wt, kw):
            v = verts.detach().cpu().numpy().astype(np.float64)
            m = complex(float(m_re), float(m_im))
            gv = None
            if verts.requires_grad:
                loss, gv, _ = adjoint_grad_vertices(bctx, v, tris, ka, m, target, wt, **kw)
            loss_m, gm, _ = adjoint_grad(bctx, v, tris, ka, m, target, wt, **kw)
            if gv is None:
                loss = loss_m
            fctx.gv = None if gv is None else torch.from_numpy(gv).to(verts.dtype)
            fctx.gm = torch.from_numpy(gm)
            return torch.tensor(loss, dtype=torch.float64)

        @staticmethod
        def backward(fctx, gout):
            gv = None if fctx.gv is None else gout * fctx.gv
            return gv, gout * fctx.gm[0], gout * fctx.gm[1], None, None, None, None, None, None

    return MuellerMisfit


_MISFIT = None


def mueller_misfit(ctx: Context, verts, tris, ka, m_re, m_im, target, wt=None, **kw):
    """Differentiable M11 misfit for torch: verts (nv, 3) and m_re, m_im are
    float64 torch tensors (CPU), the loss a 0-d tensor whose backward() fills
    verts.grad (when verts requires it) and m_re.grad, m_im.grad from one
    forward and one adjoint solve each (bem_adjoint_grad_vertices,
    bem_adjoint_grad).  target: one value per scattering angle; **kw as
    dense_run (orient, ...)."""
    global _MISFIT
    if _MISFIT is None:
        _MISFIT = _misfit_function()
    target = np.ascontiguousarray(target, dtype=np.float64)
    return _MISFIT.apply(verts, m_re, m_im, ctx, tris, ka, target, wt, kw)


def c5_mesh(seed, refinements=3, rms=0.05, lmax=6, slope=2.0):
    """The seeded shape-gradient workload: an icosphere with a radial
    displacement r -> r (1 + g(rhat)), g a Gaussian random field of real
    spherical harmonics of degree 1..lmax (i.i.d. normal coefficients with
    variance (l + 1)^-slope), scaled to RMS `rms` over the vertices."""
    from scipy.special import sph_harm_y
    v, t = icosphere(1.0, refinements)
    rng = np.random.default_rng(seed)
    r = np.linalg.norm(v, axis=1)
    th = np.arccos(np.clip(v[:, 2] / r, -1.0, 1.0))
    ph = np.arctan2(v[:, 1], v[:, 0])
    g = np.zeros(len(v))
    for ell in range(1, lmax + 1):
        sd = (ell + 1.0) ** (-slope / 2.0)
        for mm in range(-ell, ell + 1):
            y = sph_harm_y(ell, abs(mm), th, ph)
            yr = y.real if mm == 0 else np.sqrt(2.0) * (y.real if mm > 0 else y.imag)
            g += rng.standard_normal() * sd * yr
    g *= rms / np.sqrt(np.mean(g ** 2))
    return v * (1.0 + g)[:, None], t


def c4_particles(seed, count=64, orient=(4, 4, 1), ntheta=181, precision=PREC_FP64):
    """The seeded batched-particle workload: hex prisms with aspect ratio
    U[0.5, 2], refinement 2 or 3 (2N = 1152 / 4608), ka U[1, 5], Re m
    U[1.30, 1.60], Im m log-uniform in [1e-6, 1e-2], 4 x 4 x 1 orientations."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        ar = rng.uniform(0.5, 2.0)
        ref = int(rng.integers(2, 4))
        ka = rng.uniform(1.0, 5.0)
        m = complex(rng.uniform(1.30, 1.60), 10.0 ** rng.uniform(-6.0, -2.0))
        v, t = hex_prism(ar, ref)
        out.append(dict(verts=v, tris=t, ka=ka, m=m, orient=orient, ntheta=ntheta, precision=precision,
                        meta={"aspect_ratio": ar, "refinements": ref}))
    return out


def cgemm_tf32x3(ctx: Context, A, B, C, b_rowmajor=True, c_colmajor=False):
    """C -= A B on the tensor cores, torch complex64 device tensors: three
    products of two-part operands, FP16 parts after power-of-two row / column
    scaling (default) or TF32 parts (set_option(ctx, "tensor_split", 0)).
    A: (M, K) row-major; B: (K, N) row-major if b_rowmajor else given as its
    transpose (N, K) row-major; C: (M, N) row-major, or (N, M) if c_colmajor."""
    M, K = A.shape
    if b_rowmajor:
        N = B.shape[1]
    else:
        N = B.shape[0]
    ctx.check(lib().bem_cgemm_tf32x3(ctx.h, M, N, K, _dptr(A), A.stride(0), _dptr(B), B.stride(0),
                                     int(bool(b_rowmajor)), _dptr(C), C.stride(0),
                                     int(bool(c_colmajor))))
    return C


def set_tensor_cores(ctx: Context, enable: bool):
    ctx.check(lib().bem_ctx_set_tensor_cores(ctx.h, int(bool(enable))))


def set_symmetric(ctx: Context, mode: int):
    """1 (default): FP32 L D L^T without pivoting for symmetric-structured Z
    (PMCHWT); 0: always LU with partial pivoting."""
    ctx.check(lib().bem_ctx_set_symmetric(ctx.h, int(mode)))


def set_option(ctx: Context, name: str, value: int):
    """Named switches of bem_ctx_set_option (include/bem_dense.h lists them)."""
    ctx.check(lib().bem_ctx_set_option(ctx.h, name.encode(), int(value)))


def set_residual_digits(ctx: Context, digits: int):
    """Digits of the int8 refinement residual (0: FP64 GEMM residual)."""
    ctx.check(lib().bem_ctx_set_residual_digits(ctx.h, int(digits)))


def mueller_noalloc_dev(geom: Geometry, X, RT, w, k_ext, eta_ext, M_out, ntheta=181,
                        gamma_mirror=False):
    """bem_farfield_mueller_noalloc: same sum as mueller_from_solutions_dev into
    the caller's device buffer M_out (torch float64, 16*ntheta), with no device
    allocation by the library (scratch is a static device array)."""
    import torch
    RT, w = _check_solutions(geom, X, RT, w)
    if not (isinstance(M_out, torch.Tensor) and M_out.dtype == torch.float64 and M_out.is_cuda
            and M_out.device.index == geom.ctx.device and M_out.is_contiguous()
            and M_out.numel() >= 16 * int(ntheta)):
        raise ValueError("M_out must be a contiguous float64 device tensor of at least 16*ntheta elements")
    k = complex(k_ext)
    geom.ctx.check(lib().bem_farfield_mueller_noalloc(
        geom.ctx.h, geom.h, _dptr(X), X.stride(0), _ptr(RT), _ptr(w), RT.shape[0], k.real, k.imag,
        float(eta_ext), int(ntheta), int(bool(gamma_mirror)), _dptr(M_out)))
    return M_out
