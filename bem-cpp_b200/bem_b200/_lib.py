"""ctypes binding of libbemdense.so (declared in include/bem_dense.h).

The library is built in-tree (``make -C bem-cpp_b200`` or
``__graft_entry__.build()``).  There is no fallback: if it is missing, every
call raises ``BemLibraryMissing``.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libbemdense.so")

STATUS = {0: "BEM_OK", 1: "BEM_ERR_INVALID", 2: "BEM_ERR_CUDA", 3: "BEM_ERR_OOM",
          4: "BEM_ERR_SINGULAR", 5: "BEM_ERR_NOCONV", 6: "BEM_ERR_TIMEOUT",
          7: "BEM_ERR_NODEVICE"}

PREC_FP64 = 0
PREC_FP32_REFINE = 1
ASM_GSMOOTH_EXACT = 1


class BemLibraryMissing(RuntimeError):
    pass


class BemError(RuntimeError):
    def __init__(self, status, msg=""):
        self.status = status
        super().__init__(f"{STATUS.get(status, status)}: {msg}")


class SolveStats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("converged", C.c_int),
                ("max_rel_update", C.c_double), ("max_rel_residual", C.c_double),
                ("est_rel_error", C.c_double),
                ("t_factor_ms", C.c_double), ("t_solve_ms", C.c_double),
                ("t_refine_ms", C.c_double), ("update_hist", C.c_double * 12),
                ("factorization", C.c_int), ("verified_columns", C.c_int),
                ("verified_rel_error", C.c_double), ("exact_residual_sweeps", C.c_int),
                ("info", C.c_int)]

    def as_dict(self):
        d = {f: getattr(self, f) for f, _ in self._fields_}
        d["update_hist"] = [self.update_hist[i] for i in range(min(12, self.iterations))]
        return d


class GmresStats(C.Structure):
    _fields_ = [("converged", C.c_int), ("n_unconverged", C.c_int),
                ("max_iterations", C.c_int), ("total_iterations", C.c_int),
                ("max_cycles", C.c_int), ("matvecs", C.c_int),
                ("max_rel_residual", C.c_double), ("t_ms", C.c_double)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


PRECOND_NONE, PRECOND_DIAG, PRECOND_BLOCK_DIAG, PRECOND_LU = 0, 1, 2, 3

SOLVER_LU, SOLVER_GMRES_AEXT = 0, 1


class Problem(C.Structure):
    _fields_ = [("verts", C.c_void_p), ("nv", C.c_int), ("tris", C.c_void_p), ("nt", C.c_int),
                ("ka", C.c_double), ("m_re", C.c_double), ("m_im", C.c_double),
                ("quad_order", C.c_int), ("single", C.c_int),
                ("n_alpha", C.c_int), ("n_beta", C.c_int), ("n_gamma", C.c_int),
                ("beta_sym", C.c_int), ("gamma_sym", C.c_int), ("gamma_mirror", C.c_int),
                ("orient_i0", C.c_int), ("orient_i1", C.c_int), ("ntheta", C.c_int),
                ("precision", C.c_int), ("refine_tol", C.c_double), ("max_refine", C.c_int),
                ("asm_flags", C.c_uint), ("orient_tol", C.c_double),
                ("solver", C.c_int), ("gmres_tol", C.c_double), ("gmres_restart", C.c_int),
                ("gmres_maxiter", C.c_int)]


class Result(C.Structure):
    _fields_ = [("mueller", C.c_void_p), ("t_assembly_s", C.c_double),
                ("t_solve_s", C.c_double), ("t_farfield_s", C.c_double),
                ("t_total_s", C.c_double), ("N", C.c_int), ("n_orient", C.c_int),
                ("stats", SolveStats), ("per_orient_mueller", C.c_void_p),
                ("per_orient_weight", C.c_void_p), ("n_computed", C.c_int),
                ("t_setup_s", C.c_double), ("t_release_s", C.c_double),
                ("gmres", GmresStats)]


_P = C.c_void_p
_I = C.c_int
_D = C.c_double
_L = C.c_int64
_IP = C.POINTER(C.c_int)

# name -> (restype, argtypes); every int-returning function is a status
SIGNATURES = {
    "bem_ctx_create": (_I, [_I, C.POINTER(_P)]),
    "bem_ctx_destroy": (_I, [_P]),
    "bem_ctx_set_stream": (_I, [_P, _P]),
    "bem_ctx_synchronize": (_I, [_P]),
    "bem_last_error": (C.c_char_p, [_P]),
    "bem_ctx_launch_count": (_L, [_P]),
    "bem_version": (C.c_char_p, []),
    "bem_selftest_bounded_wait": (_I, [_P, C.c_int64, _I]),
    "bem_ctx_profile": (_I, [_P, _I]),
    "bem_ctx_set_tensor_cores": (_I, [_P, _I]),
    "bem_ctx_set_residual_digits": (_I, [_P, _I]),
    "bem_ctx_set_symmetric": (_I, [_P, _I]),
    "bem_ctx_set_option": (_I, [_P, C.c_char_p, _I]),
    "bem_lu_residual_dev": (_I, [_P, _P, _P, _L, _P, _L, _P, _L, _I, _I]),
    "bem_cgemm_tf32x3": (_I, [_P, _I, _I, _I, _P, _L, _P, _L, _I, _P, _L, _I]),
    "bem_ctx_profile_read": (_I, [_P, _I, C.POINTER(_L), C.POINTER(_D), C.POINTER(_D),
                                  C.POINTER(_D)]),
    "bem_mesh_icosphere": (_I, [_D, _I, _IP, _IP, _P, _P]),
    "bem_mesh_hex_prism": (_I, [_D, _I, _IP, _IP, _P, _P]),
    "bem_mesh_subdivide_flat": (_I, [_P, _I, _P, _I, _IP, _IP, _P, _P]),
    "bem_mesh_load_obj": (_I, [C.c_char_p, _IP, _IP, _P, _P, _IP, _IP]),
    "bem_mesh_normalize": (_I, [_P, _I, _P, _I, C.POINTER(_D)]),
    "bem_mesh_volume": (_D, [_P, _I, _P, _I]),
    "bem_mesh_dmax": (_D, [_P, _I]),
    "bem_rwg_build": (_I, [_P, _I, _P, _I, _IP, _P, _P, _P, _P, _P, _P, _P]),
    "bem_tri_quadrature": (_I, [_I, _IP, _P, _P]),
    "bem_orientations": (_I, [_I, _I, _I, _I, _I, _I, _I, _IP, _P, _P]),
    "bem_gauss_legendre": (_I, [_I, _P, _P]),
    "bem_geom_create": (_I, [_P, _P, _I, _P, _I, _I, C.POINTER(_P), _IP]),
    "bem_geom_create_rwg": (_I, [_P, _P, _I, _P, _I, _I, _P, _P, _P, _P, _P, _P, _P, _I,
                                 C.POINTER(_P)]),
    "bem_geom_free": (_I, [_P]),
    "bem_geom_size": (_I, [_P]),
    "bem_geom_set_vertices": (_I, [_P, _P, _P]),
    "bem_assemble_pmchwt_dev": (_I, [_P, _P, _D, _D, _D, _D, _D, _D, C.c_uint, _P, _L]),
    "bem_assemble_LK_dev": (_I, [_P, _P, _D, _D, C.c_uint, _P, _P, _L]),
    "bem_assemble_aext_dev": (_I, [_P, _P, _D, _D, _D, C.c_uint, _P, _L]),
    "bem_precond_create": (_I, [_P, _I, _P, _I, _L, _I, _P, C.POINTER(_P)]),
    "bem_precond_free": (_I, [_P]),
    "bem_gmres_solve_dev": (_I, [_P, _P, _I, _L, _P, _P, _L, _P, _L, _I, _I, _D, _I, _P, _P,
                                 C.POINTER(GmresStats)]),
    "bem_assemble_L_K": (_I, [_P, _P, _I, _P, _I, _D, _D, _I, _P, _P]),
    "bem_assemble_pmchwt": (_I, [_P, _P, _I, _P, _I, _D, _D, _D, _D, _D, _D, _I, _P, _P, _P]),
    "bem_rhs_planewave_dev": (_I, [_P, _P, _D, _D, _D, _P, _I, _P, _L]),
    "bem_rhs_planewave": (_I, [_P, _P, _D, _D, _D, _P, _P, _P]),
    "bem_lu_factor_dev": (_I, [_P, _P, _I, _L, _I, C.POINTER(_P), _IP]),
    "bem_lu_solve_dev": (_I, [_P, _P, _P, _L, _P, _L, _I, _D, _I, C.POINTER(SolveStats)]),
    "bem_lu_free": (_I, [_P]),
    "bem_lu_factorize": (_I, [_P, _P, _I, _P, _IP]),
    "bem_lu_solve": (_I, [_P, _P, _P, _I, _P, _I]),
    "bem_lu_solve_full": (_I, [_P, _P, _I, _P, _I, _I, C.POINTER(SolveStats)]),
    "bem_farfield_batch": (_I, [_P, _P, _P, _P, _P, _D, _D, _D, _I, _I, _I, _P]),
    "bem_farfield_mueller_dev": (_I, [_P, _P, _P, _L, _P, _P, _I, _D, _D, _D, _I, _I, _P, _P]),
    "bem_farfield_mueller_noalloc": (_I, [_P, _P, _P, _L, _P, _P, _I, _D, _D, _D, _I, _I, _P]),
    "bem_amplitude_to_mueller": (_I, [_P, _P, _P, _P, _I, _P]),
    "bem_dense_run": (_I, [_P, C.POINTER(Problem), C.POINTER(Result)]),
    "bem_batch_run": (_I, [_P, C.POINTER(Problem), _I, C.POINTER(Result), C.POINTER(_I)]),
    "bem_adjoint_grad": (_I, [_P, C.POINTER(Problem), _P, _P, C.POINTER(_D), _P, _P]),
    "bem_adjoint_grad_vertices": (_I, [_P, C.POINTER(Problem), _P, _P, C.POINTER(_D), _P, _P]),
}

_lib = None


def lib():
    """Loads the library once; raises BemLibraryMissing if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise BemLibraryMissing(
                f"{LIB_PATH} not built: run `make -C bem-cpp_b200` (no CPU fallback exists)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            try:
                fn = getattr(L, name)
            except AttributeError:
                continue  # reported by missing_symbols()
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def missing_symbols():
    """Entry points of include/bem_dense.h that the built library lacks."""
    L = lib()
    return [n for n in SIGNATURES if not hasattr(L, n)]


def check(status, ctx=None):
    if status != 0:
        msg = ""
        if ctx is not None:
            msg = (lib().bem_last_error(ctx) or b"").decode(errors="replace")
        raise BemError(status, msg)
