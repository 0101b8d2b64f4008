/*
 * bem_dense.h -- C ABI of libbemdense.so, a B200-native (sm_100a) implementation
 * of the dense PMCHWT path of BEM-CPP: RWG Galerkin assembly of the 2N x 2N
 * system, complex LU with a multi-RHS solve (FP64, or FP32 factors with FP64
 * iterative refinement), and the far-field / Mueller reduction.
 *
 * Plain C types only.  Complex numbers are interleaved (re, im) doubles, the
 * layout of std::complex<double> / cuDoubleComplex.  Matrices named Z are
 * row-major n x n (the reference's Z[i*n + j]); right-hand sides and solutions
 * are column-major n x nrhs (column c at B[c*n]), as in the reference.
 *
 * Every entry point returns a bem_status.  Nothing calls exit(); the message of
 * the last failure on a context is available from bem_last_error().
 *
 * Reference interfaces each entry point replaces are cited as
 * file:line of KirillSalnikov/BEM-CPP.
 */
#ifndef BEM_DENSE_H
#define BEM_DENSE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum bem_status {
    BEM_OK = 0,
    BEM_ERR_INVALID = 1,    /* bad argument (size, pointer, order, option) */
    BEM_ERR_CUDA = 2,       /* CUDA runtime / launch failure */
    BEM_ERR_OOM = 3,        /* device allocation failed */
    BEM_ERR_SINGULAR = 4,   /* zero pivot; the LU info is returned separately */
    BEM_ERR_NOCONV = 5,     /* iterative refinement did not reach the tolerance */
    BEM_ERR_TIMEOUT = 6,    /* a bounded device-side wait gave up */
    BEM_ERR_NODEVICE = 7    /* no usable sm_100 device */
} bem_status;

typedef enum bem_precision {
    BEM_PREC_FP64 = 0,         /* complex128 LU and solves */
    BEM_PREC_FP32_REFINE = 1   /* complex64 LU (tensor-core updates, FP16 or TF32 operand parts) + FP64 refinement */
} bem_precision;

/* Assembly flags */
#define BEM_ASM_GSMOOTH_EXACT 1u  /* cancellation-free G_smooth limit ik/(4 pi) at R = 0
                                     (default: the reference's exp(ikR)/(4piR) - 1/(4piR)
                                     with R clamped to 1e-15, assembly.cu:63-77) */

typedef struct bem_ctx bem_ctx;        /* device, stream, workspace */
typedef struct bem_geom bem_geom;      /* device-resident mesh + RWG quadrature data */
typedef struct bem_lu bem_lu;          /* device-resident factorisation */

/* ---------------------------------------------------------------- context */

/* Opens a context on `device` (an sm_100 GPU).  One context per host thread. */
int bem_ctx_create(int device, bem_ctx** out);
int bem_ctx_destroy(bem_ctx* ctx);
/* Kernels of this context run on `stream` (a cudaStream_t).  A new context
 * uses a private non-blocking stream; NULL selects the legacy default stream. */
int bem_ctx_set_stream(bem_ctx* ctx, void* stream);
int bem_ctx_synchronize(bem_ctx* ctx);
const char* bem_last_error(const bem_ctx* ctx);
/* Number of kernel launches issued by this context so far. */
int64_t bem_ctx_launch_count(const bem_ctx* ctx);

/* Per-kernel-class device timing: CUDA events on the context's stream around
 * every launch of a class.  bem_ctx_profile(ctx, 1) clears the counters and
 * starts recording, 0 stops.  Classes: 0 LU trailing update, 1 triangular
 * solve block updates, 2 FP64 refinement residual, 3 panel factorisation,
 * 4 assembly, 5 far field / Mueller, 6 the FP64 residual of the columns
 * checked after the refinement, 7 triangular solves with a diagonal block,
 * 8 row interchanges and permutations, 9 updates inside a block column (the
 * pivoted LU's sub-panel GEMMs, L21 of the L D L^T diagonal blocks); class 3
 * is then the panel kernels and the L D L^T diagonal blocks alone.  flops /
 * bytes are the algorithmic
 * counts of the recorded launches (complex GEMM: 8 M N K flop). */
int bem_ctx_profile(bem_ctx* ctx, int enable);
/* FP32 factorisation / solve updates on the tensor cores (three tcgen05
 * products of two-part operands, default 1) or on the CUDA cores (0). */
int bem_ctx_set_tensor_cores(bem_ctx* ctx, int enable);
/* FP64 refinement residual of BEM_PREC_FP32_REFINE factorisations made after
 * this call: digits = 0 computes B - Z X with the FP64 (DMMA) complex GEMM;
 * digits = 2..8 with the int8 tensor-core Ozaki scheme using that many 7-bit
 * digits per entry (default 7, 49 bits; needs 2 digits x n^2 x digits bytes
 * more device memory, and falls back to the FP64 GEMM when that is short). */
int bem_ctx_set_residual_digits(bem_ctx* ctx, int digits);
/* FP32 factorisation of BEM_PREC_FP32_REFINE systems whose Z, or Z diag(I, -I)
 * (the PMCHWT structure: symmetric L and K blocks), is exactly symmetric:
 * mode 1 (default) factors that matrix as L D L^T without pivoting (half the
 * flops of LU, checked bitwise at factor time), falling back to partial
 * pivoting on a zero pivot or when the refinement does not converge; mode 0
 * always uses LU with partial pivoting. */
int bem_ctx_set_symmetric(bem_ctx* ctx, int mode);
/* Kernel-shape switches, mainly for measurement: "persistent_gemm" (1, default: persistent tensor-core GEMM; 0: one CTA per
 * tile), "residual_pace_epoch" / "residual_pace_lead" (32 / 2: the int8
 * residual's CTAs report every 32 K slabs and wait, softly, when more than 2
 * epochs ahead of the grid average, so a wave shares its digit rows in L2;
 * epoch 0 turns the pacing off), "factor_superblock" / "solve_superblock"
 * (4, default: the L D L^T factorisation and solves update with four
 * 256-wide blocks at once, K = 1024; 1..3: that many blocks, K = 256 per
 * block),
 * "gmres_digits" (0, default: GMRES
 * products with Z on the FP64 GEMM; 2..8: int8 Ozaki digits),
 * "cache_factor_memory" (0, default; 1: the FP32 factors and int8 digit planes
 * of a freed factorisation stay allocated on this context's device and are
 * reused by the next factorisation of the same order, so a loop of solves of
 * one size allocates them once; the kept memory counts against the device
 * until the option is set back to 0, which frees it, or until an allocation
 * of this library fails, which frees it and retries; the dense pipeline's
 * operator, right-hand-side and geometry buffers are cached the same way, and
 * bem_batch_run turns the cache on for its duration), "gemm_group_m" (16,
 * default: row tiles per raster group of the persistent tensor-core GEMM),
 * "assembly_kernel" (0, default: triangle-pair moments over Morton-ordered
 * tiles; 1: one thread per RWG pair, the reference's organisation),
 * "farfield_kernel" (0, default: phases shared by the RWG halves of a
 * triangle; 1: per RWG-half point), "batch_buckets" (1, default: bem_batch_run batches FP64 particles of one
 * system size -- one assembly pass, one batched LU and one batched solve per
 * size; 0: one particle at a time), "lu_autotune" (1, default: the batched
 * LU's block and panel widths are chosen by timing the candidates once per
 * (size, batch) in the process; 0: 256 / 16, the single LU's shape, whose
 * factors are bitwise those of bem_lu_factor_dev), "gradient_method" (0,
 * default: the adjoint gradients contract the operator's derivative in
 * kernels; 1: central differences of reassembled operators, for checking),
 * "panel_clusters" (1, default: the sub-panels of the pivoted LU that fit the
 * shared memory of one cluster of at most 8 CTAs -- all of them up to order
 * ~6000 -- are factored by one thread-block cluster per matrix, one cluster
 * barrier per column; 0: every sub-panel on the cooperative grid, one grid
 * barrier per column; both give the same pivots and factors),
 * "fp64_gemm_3m" (1, default: the complex FP64 GEMMs of the pivoted LU, its
 * solves and the FP64 residual take three real products per complex product,
 * Re = Ar Br - Ai Bi, Im = (Ar + Ai)(Br + Bi) - Ar Br - Ai Bi, on the FP64
 * tensor path: 6MNK instead of 8MNK multiply-adds, error normwise at the FP64
 * unit roundoff; 0: four real products),
 * "residual_x_digits" (2, default: the refinement rounds its first iterate
 * (the FP32 solve's) and each correction it sums with the int8 residual's
 * update form to their first 2 digits of 7 bits below their column's
 * largest entry, and keeps the rounded values, so the int8 residual needs
 * only the digit pairs of those digits -- 13 instead of 28 for the first
 * residual, 11 instead of 21 for a 6-digit update -- and stays exact for the
 * iterate it belongs to; the rounding, 2^-14 of the column's largest entry,
 * is below the FP32 solve's own error and the next sweep removes it; 0:
 * every digit, 1..7: that many),
 * "lu_u12_slabs" (1, default: the FP64 LU forms U12 = L11^-1 A12 of
 * every 256-column block by 64-row slabs, each solved by the block
 * triangular solve and followed by the GEMM update of the slabs below on
 * the FP64 tensor path -- the same substitution regrouped, three quarters
 * of its flops in the GEMM; 0: one block triangular solve of 256 rows),
 * "solve_block_inverse" (1, default: the FP32 L D L^T factorisation also
 * keeps -L11^-1 of each 256-row diagonal block (n^2 / 256 complex64, 8 n^2 /
 * 256 bytes), and its solves apply the diagonal blocks as tensor-core
 * products with them; 0, or without memory for them: block triangular
 * solves; set before the factorisation),
 * "ldlt_cluster_diag" (1, default: the FP32 L D L^T factors each 256 x 256
 * diagonal block on one cluster of 8 CTAs that holds the block in
 * distributed shared memory, 32 rows per CTA; 0, or where such a cluster
 * cannot be resident: on one CTA; both take every entry through the same
 * operations in the same order),
 * "gemm_pairs" (1, default: the FP16-part tensor-core GEMM on 256-row tiles
 * of CTA pairs, tcgen05.mma.cta_group::2, each CTA loading half of a tile's
 * B operand; 0: 128-row tiles, one CTA each),
 * "verify_columns" (64, default: after the refinement converges, the error of
 * 64 columns is measured with an FP64 residual, see bem_lu_solve_dev; -1:
 * every column; 0: no check), "tensor_split" (1, default: FP32
 * operands of the tensor-core GEMM split into two FP16 parts after a
 * power-of-two scale per operand row / column that brings its largest part
 * into [2^14, 2^15), kind::f16 at twice the TF32 rate, the persistent GEMM
 * only; 0: into two TF32 parts, kind::tf32.  Both give FP32-class products;
 * with FP16 parts an entry below about 2^-18 of its row's (column's) largest
 * keeps fewer than 22 significant bits).  Unknown names give
 * BEM_ERR_INVALID. */
int bem_ctx_set_option(bem_ctx* ctx, const char* name, int value);
int bem_ctx_profile_read(bem_ctx* ctx, int cls, int64_t* launches, double* ms, double* flops,
                         double* bytes);
const char* bem_version(void);
/* The failure path of a bounded device-side wait, without a fault: one
 * thread waits on a device flag for at most `cycles` SM clock cycles
 * (0..4e9).  set_flag = 0: nothing sets the flag, the wait runs out and the
 * call returns BEM_ERR_TIMEOUT with the context still usable; set_flag = 1:
 * BEM_OK.  No counterpart in the reference (its CUDA errors exit). */
int bem_selftest_bounded_wait(bem_ctx* ctx, int64_t cycles, int set_flag);

/* ----------------------------------------------------- geometry (host) */
/* Meshes are returned through caller buffers.  Pass NULL buffers to query
 * the sizes first. */

/* icosphere(radius, refinements) -- mesh.cpp:11-68 */
int bem_mesh_icosphere(double radius, int refinements, int* nv, int* nt,
                       double* verts, int* tris);
/* hex_prism(aspect_ratio, refinements) -- mesh.cpp:102-154 */
int bem_mesh_hex_prism(double aspect_ratio, int refinements, int* nv, int* nt,
                       double* verts, int* tris);
/* subdivide_flat(mesh) -- mesh.cpp:70-100 (out buffers sized by a NULL query) */
int bem_mesh_subdivide_flat(const double* verts, int nv, const int* tris, int nt,
                            int* nv_out, int* nt_out, double* verts_out, int* tris_out);
/* load_obj(filename) -- mesh.cpp:156-250; removes degenerate triangles and
 * counts non-manifold edges into *n_nonmanifold (may be NULL). */
int bem_mesh_load_obj(const char* filename, int* nv, int* nt, double* verts, int* tris,
                      int* n_degenerate, int* n_nonmanifold);
/* normalize_mesh / mesh_volume / mesh_dmax -- mesh.cpp:252-294 */
int bem_mesh_normalize(double* verts, int nv, const int* tris, int nt, double* a_eq);
double bem_mesh_volume(const double* verts, int nv, const int* tris, int nt);
double bem_mesh_dmax(const double* verts, int nv);

/* build_rwg(mesh) -- rwg.cpp:5-43: interior edges in (min,max) vertex order.
 * Arrays of length N; free_p / free_m are 3N doubles.  NULL arrays = size query. */
int bem_rwg_build(const double* verts, int nv, const int* tris, int nt, int* N,
                  int* tri_p, int* tri_m, double* free_p, double* free_m,
                  double* length, double* area_p, double* area_m);

/* tri_quadrature(order) -- quadrature.h:14-70.  pts: 2*npts (l1, l2), wts: npts. */
int bem_tri_quadrature(int order, int* npts, double* pts, double* wts);

/* generate_orientations (+ optional sort_orientations_nearest) -- orient.cpp:73-163.
 * RT: 9 doubles per orientation (row-major R^T), w: weights. NULL = size query. */
int bem_orientations(int n_alpha, int n_beta, int n_gamma, int beta_sym, int gamma_sym,
                     int gamma_mirror, int sort_nearest, int* count, double* RT, double* w);
/* gauss_legendre(n) -- orient.cpp:39-70 */
int bem_gauss_legendre(int n, double* nodes, double* weights);

/* ----------------------------------------------------- device geometry */

/* Uploads a mesh and builds its RWG basis and quadrature data on the device
 * (precompute_half, assembly.cu:150-201; FFCache::init, farfield.cu:9-52).
 * *N receives the number of RWG functions (system size 2N). */
int bem_geom_create(bem_ctx* ctx, const double* verts, int nv, const int* tris, int nt,
                    int quad_order, bem_geom** out, int* N);
/* Same with an explicit RWG basis (arrays of length N; free_p / free_m 3N
 * doubles), for callers that built theirs with build_rwg (rwg.h:18). */
int bem_geom_create_rwg(bem_ctx* ctx, const double* verts, int nv, const int* tris, int nt, int N,
                        const int* tri_p, const int* tri_m, const double* free_p, const double* free_m,
                        const double* length, const double* area_p, const double* area_m,
                        int quad_order, bem_geom** out);
int bem_geom_free(bem_geom* g);
int bem_geom_size(const bem_geom* g);
/* Moves the vertices of a geometry made by bem_geom_create (verts: nv x 3
 * doubles, same mesh topology) in place: the position-dependent device data
 * is recomputed and copied into the same allocation in the stream order of
 * ctx, keeping the RWG order and the assembly tiles; right-hand sides and far
 * field equal those of a geometry created from the moved mesh, the operator
 * to rounding (each symmetric pair is computed in the orientation of the kept
 * tiles).  For loops over shapes of one mesh (shape gradients,
 * optimisation); no reference counterpart.
 * BEM_ERR_INVALID for a geometry made by bem_geom_create_rwg. */
int bem_geom_set_vertices(bem_ctx* ctx, bem_geom* g, const double* verts);

/* --------------------------------------------------------------- assembly */

/* Device-resident PMCHWT matrix (pmchwt.cu:6-56 with assemble_L_K_cuda,
 * assembly.cu:328-505, for both media in one pass):
 *   Z = [[eta_e L_e + eta_i L_i, -(K_e + K_i)], [K_e + K_i, L_e/eta_e + L_i/eta_i]]
 * Z_dev: row-major 2N x 2N complex128 with leading dimension ldz (elements). */
int bem_assemble_pmchwt_dev(bem_ctx* ctx, const bem_geom* g,
                            double kext_re, double kext_im, double kint_re, double kint_im,
                            double eta_ext, double eta_int, unsigned flags,
                            void* Z_dev, int64_t ldz);
/* Device-resident L and K for one wavenumber (assemble_L_K_cuda, assembly.h:11-13):
 * row-major N x N complex128, leading dimension ld. */
int bem_assemble_LK_dev(bem_ctx* ctx, const bem_geom* g, double k_re, double k_im,
                        unsigned flags, void* L_dev, void* K_dev, int64_t ld);
/* Exterior-only PMCHWT (build_aext_preconditioner, bem_core.py:1071-1090):
 *   A_ext = [[eta_e L_e, -K_e], [K_e, L_e/eta_e]]
 * the preconditioner of the A_ext GMRES (A_ext^-1 Z = I + A_ext^-1 A_int with
 * A_int compact).  Z_dev: row-major 2N x 2N complex128, leading dimension ldz. */
int bem_assemble_aext_dev(bem_ctx* ctx, const bem_geom* g, double kext_re, double kext_im,
                          double eta_ext, unsigned flags, void* Z_dev, int64_t ldz);
/* Host-buffer mirrors: assemble_L_K_cuda (assembly.h:11-13) and assemble_pmchwt
 * (pmchwt.h:12-18).  L_ext / K_ext of the latter may be NULL. */
int bem_assemble_L_K(bem_ctx* ctx, const double* verts, int nv, const int* tris, int nt,
                     double k_re, double k_im, int quad_order, double* L, double* K);
int bem_assemble_pmchwt(bem_ctx* ctx, const double* verts, int nv, const int* tris, int nt,
                        double kext_re, double kext_im, double kint_re, double kint_im,
                        double eta_ext, double eta_int, int quad_order,
                        double* Z, double* L_ext, double* K_ext);

/* ------------------------------------------------------------ excitation */

/* Plane-wave right-hand sides for a batch of orientations (rhs.cpp:6-64,
 * main.cpp:739-751): column 2o = par (E0 = RT x), 2o+1 = perp (E0 = RT y),
 * k_hat = RT z.  RT: host, 9 doubles per orientation.  B_dev: column-major
 * 2N x (2 n_orient) complex128, leading dimension ldb. */
int bem_rhs_planewave_dev(bem_ctx* ctx, const bem_geom* g, double k_re, double k_im,
                          double eta_ext, const double* RT, int n_orient,
                          void* B_dev, int64_t ldb);
/* One plane wave, host output (compute_rhs_planewave, rhs.h:11-15). */
int bem_rhs_planewave(bem_ctx* ctx, const bem_geom* g, double k_re, double k_im,
                      double eta_ext, const double* E0, const double* k_hat, double* b);

/* -------------------------------------------------------------------- LU */

typedef struct bem_solve_stats {
    int iterations;          /* refinement sweeps run (0 for FP64) */
    int converged;           /* 1 when the error estimate met the tolerance */
    double max_rel_update;   /* max over columns of max|dX| / max|X| in the last sweep */
    double max_rel_residual; /* max over columns of max|B - Z X| / (||Z||_F max|X|) */
    double est_rel_error;    /* estimated max-column relative error of the returned X */
    double t_factor_ms, t_solve_ms, t_refine_ms;
    double update_hist[12];  /* max relative update of sweeps 1..12 */
    int factorization;       /* FP32 factors used: 0 LU with partial pivoting, 1 L D L^T of Z,
                                2 L D L^T of Z diag(I, -I); -1 FP64 */
    int verified_columns;    /* columns whose error was measured at convergence (option verify_columns) */
    double verified_rel_error; /* max over those columns of max|e| / max|x|, e = (factors)^-1 (B - Z X)
                                  with B - Z X in the FP64 GEMM */
    int exact_residual_sweeps; /* sweeps that fell back to the FP64 GEMM residual, after a check showed
                                  the int8 residual's floor above the tolerance (or without its memory) */
    int info;                /* bem_lu_solve_full: the LU's info (0, or the 1-based index of the first
                                zero pivot, with BEM_ERR_SINGULAR) */
} bem_solve_stats;

/* Factorises the row-major n x n complex128 matrix Z_dev (leading dimension
 * ldz) with partial pivoting.  FP64: Z_dev is overwritten by the factors.
 * FP32_REFINE: Z_dev is kept (the refinement residual needs it; it must stay
 * valid until bem_lu_free) and complex64 factors are made in new memory.
 * *info: 0, or k > 0 when U(k,k) is exactly zero (1-based, LAPACK convention). */
int bem_lu_factor_dev(bem_ctx* ctx, void* Z_dev, int n, int64_t ldz, int precision,
                      bem_lu** out, int* info);
/* X = Z^-1 B for nrhs columns (column-major, leading dimensions ldb / ldx; X may
 * alias B).  FP32_REFINE refines in FP64 (residual B - Z X with the FP64 Z,
 * correction through the FP32 factors) until the estimated relative error of
 * every column is below `tol` (default 1e-11 when tol <= 0), or max_iter
 * sweeps (default 10) were run (BEM_ERR_NOCONV).  The estimate is the larger
 * of two: rho/(1-rho) times the last relative update, rho the observed
 * contraction (how far the sweeps are from their limit), and the error
 * measured directly at that point on the columns of the option
 * verify_columns (default 64, -1 all, 0 none; a sample takes half its
 * columns evenly spaced and half where the last sweep's relative update was
 * largest): the FP64-GEMM residual of each, solved through the factors, with
 * the sampled maximum tripled for the columns not checked (and the checked
 * ones taken 10 % above their measured error).  The second term sees the
 * floor that the int8 residual's digit truncation leaves, which the updates
 * cannot; when it is above tol the remaining sweeps compute the residual in
 * the FP64 GEMM (stats->exact_residual_sweeps) and the check is repeated. */
int bem_lu_solve_dev(bem_ctx* ctx, bem_lu* lu, const void* B_dev, int64_t ldb,
                     void* X_dev, int64_t ldx, int nrhs, double tol, int max_iter,
                     bem_solve_stats* stats);
/* R = B - Z X for a BEM_PREC_FP32_REFINE factorisation's Z (all column-major
 * complex128, R distinct from B and X).  method 0: FP64 GEMM; method 1: the
 * int8 Ozaki residual (BEM_ERR_INVALID when the factorisation has no digit
 * planes).  This is the refinement's residual step on its own. */
int bem_lu_residual_dev(bem_ctx* ctx, bem_lu* lu, const void* B_dev, int64_t ldb,
                        const void* X_dev, int64_t ldx, void* R_dev, int64_t ldr, int nrhs,
                        int method);
int bem_lu_free(bem_lu* lu);

/* Host-buffer mirrors of solver.h:11-22.  The reference factors its row-major
 * Z as a column-major Z^T (solver.cu:25-31) and solves with op = T; these keep
 * that contract: bem_lu_factorize overwrites Z with the packed LU factors of
 * the row-major Z (P Z = L U, unit L) and returns 1-based row pivots, and
 * bem_lu_solve consumes exactly that pair. */
int bem_lu_factorize(bem_ctx* ctx, double* Z, int n, int* ipiv, int* info);
int bem_lu_solve(bem_ctx* ctx, const double* Z_lu, const int* ipiv, int n, double* B, int nrhs);
int bem_lu_solve_full(bem_ctx* ctx, double* Z, int n, double* B, int nrhs, int precision,
                      bem_solve_stats* stats);

/* ------------------------------------------------------------------ GMRES */

/* Preconditioners of the reference's iterative dense solves (solve_gmres,
 * bem_core.py:1126-1183, and solve_gmres_aext, :1093-1123). */
typedef struct bem_precond bem_precond;
typedef enum bem_precond_kind {
    BEM_PRECOND_NONE = 0,        /* identity (precond=None) */
    BEM_PRECOND_DIAG = 1,        /* x / diag(Z) ('diag') */
    BEM_PRECOND_BLOCK_DIAG = 2,  /* LU of Z11 and of Z22 separately ('block_diag') */
    BEM_PRECOND_LU = 3           /* a factorisation made by the caller, e.g. of A_ext ('aext') */
} bem_precond_kind;

/* DIAG and BLOCK_DIAG are built from Z_dev (row-major n x n, leading dimension
 * ldz; BLOCK_DIAG needs n even), which must stay valid while the
 * preconditioner is used.  precision: of the BLOCK_DIAG factorisations
 * (BEM_PREC_FP64: exact solves of copies of the blocks; FP32_REFINE: FP32
 * factors, applied once without refinement).  LU: `lu`, a factorisation of
 * order n owned by the caller that must outlive the preconditioner (FP64
 * factors solve exactly; FP32 factors are applied once without refinement).
 * NONE: only n is used. */
int bem_precond_create(bem_ctx* ctx, int kind, const void* Z_dev, int n, int64_t ldz, int precision,
                       bem_lu* lu, bem_precond** out);
int bem_precond_free(bem_precond* M);

typedef struct bem_gmres_stats {
    int converged;            /* 1 when every column met ||b - Z x||_2 <= tol ||b||_2 */
    int n_unconverged;        /* columns that did not */
    int max_iterations;       /* max over columns of inner (Arnoldi) iterations */
    int total_iterations;     /* sum over columns */
    int max_cycles;           /* max over columns of restart cycles */
    int matvecs;              /* batched products with Z (each over the columns still active) */
    double max_rel_residual;  /* max over columns of ||b - Z x||_2 / ||b||_2 (FP64) */
    double t_ms;
} bem_gmres_stats;

/* GMRES(restart) for Z X = B, nrhs columns (column-major, leading dimensions
 * ldb / ldx; X distinct from B), with the algorithm of
 * scipy.sparse.linalg.gmres that the reference calls (SciPy 1.18.1): x0 = 0,
 * left preconditioning by M, modified Gram-Schmidt Arnoldi, Givens
 * rotations, an inner loop that ends when the preconditioned residual
 * estimate is below its adaptive tolerance, and restart cycles until
 * ||b - Z x||_2 <= tol ||b||_2 (recomputed in FP64) or `maxiter` cycles.  Each
 * column runs its own Krylov space; the columns share every product with Z
 * (the FP64 tensor-core GEMM, or the int8 Ozaki product with
 * bem_ctx_set_option(ctx, "gmres_digits", 2..8)).  iters / info (optional,
 * nrhs ints): inner iterations, and 0 or maxiter as scipy's info.  Columns
 * that do not converge leave stats->converged = 0 (not an error status). */
int bem_gmres_solve_dev(bem_ctx* ctx, const void* Z_dev, int n, int64_t ldz, bem_precond* M,
                        const void* B_dev, int64_t ldb, void* X_dev, int64_t ldx, int nrhs,
                        int restart, double tol, int maxiter, int* iters, int* info,
                        bem_gmres_stats* stats);

/* ------------------------------------------------------ far field, Mueller */

/* Far-field vectors Fv for coefficient columns (farfield_batch_kernel,
 * farfield.cu:100-262): coeffs_J / coeffs_M host (n_calls x N complex128),
 * r_hats host (n_orient x ndir x 3), call c uses r_hat block c/2.
 * Fv host (n_calls x ndir x 3 complex128). */
int bem_farfield_batch(bem_ctx* ctx, const bem_geom* g, const double* coeffs_J,
                       const double* coeffs_M, const double* r_hats, double k_re, double k_im,
                       double eta_ext, int n_calls, int n_orient, int ndir, double* Fv);

/* Orientation-averaged Mueller matrix from device solutions (main.cpp:757-846
 * with amplitude_to_mueller, farfield.cu:464-508): X_dev column-major
 * 2N x (2 n_orient), columns (par, perp) per orientation.  Writes
 * M_avg[16 * ntheta] (host, M[(i*4+j)*ntheta + t]) = sum_o w_o M_o / |k|^2.
 * gamma_mirror zeroes the odd blocks of each M_o (main.cpp:837-842).
 * M_orient_dev (may be NULL): device buffer of n_orient*16*ntheta doubles that
 * receives the per-orientation w_o M_o/|k|^2 terms. */
int bem_farfield_mueller_dev(bem_ctx* ctx, const bem_geom* g, const void* X_dev, int64_t ldx,
                             const double* RT, const double* w, int n_orient,
                             double k_re, double k_im, double eta_ext, int ntheta,
                             int gamma_mirror, double* M_avg, double* M_orient_dev);

/* Allocation-free variant of bem_farfield_mueller_dev, with no counterpart in
 * the reference.  For callers that cannot allocate device memory, such as
 * hosts whose device memory belongs to their own allocator (a serving stack
 * with a fixed pool).  Its only scratch (staged orientations, per-orientation
 * Mueller terms) is a file-scope device array of BEM_NOALLOC_SCRATCH_BYTES,
 * held by every GPU that loads the library until exit; the call itself
 * allocates nothing.  The scratch holds three segments, each rounded up to a
 * multiple of 256 bytes: 72 n_orient bytes (orientations), 8 n_orient bytes
 * (weights) and 128 ntheta n_orient bytes (per-orientation terms); a call
 * whose rounded sum exceeds BEM_NOALLOC_SCRATCH_BYTES is rejected with
 * BEM_ERR_INVALID: split the orientations and add the partial results (the
 * average is a weighted sum).  RT, w: host arrays as in
 * bem_farfield_mueller_dev, copied to the scratch in the context's stream
 * order: pageable memory is read before the call returns, but pinned memory
 * may still be read afterwards, so keep pinned RT and w unchanged until that
 * stream has passed the call.  M_avg_dev: caller's device buffer of
 * 16*ntheta doubles, written on the context's stream.  The first call on a device looks
 * up the scratch address (cudaGetSymbolAddress), so make that first call before
 * any stream capture begins.  All calls share the one array: calls that overlap on
 * the GPU (different streams or contexts on one device) race on it. */
#define BEM_NOALLOC_SCRATCH_BYTES (4 * 1024 * 1024)
int bem_farfield_mueller_noalloc(bem_ctx* ctx, const bem_geom* g, const void* X_dev, int64_t ldx,
                                 const double* RT, const double* w, int n_orient, double k_re, double k_im,
                                 double eta_ext, int ntheta, int gamma_mirror, double* M_avg_dev);

/* amplitude_to_mueller (farfield.cu:464-508); S*, complex128[ntheta]. */
int bem_amplitude_to_mueller(const double* S1, const double* S2, const double* S3,
                             const double* S4, int ntheta, double* M);

/* The tensor-core update used by the FP32 factorisation, exposed for direct
 * use and testing: C -= A B with complex64 device buffers.  A: M x K with K
 * contiguous (A[i*lda + k]); B: K x N, b_rowmajor ? B[k*ldb + j] :
 * B[j*ldb + k]; C: M x N, c_colmajor ? C[j*ldc + i] : C[i*ldc + j].
 * Products are hi*hi + hi*lo + lo*hi with FP32 accumulation; the parts are
 * FP16 after power-of-two row / column scaling, or TF32 with the context
 * option tensor_split = 0 (the name keeps the original TF32 form). */
int bem_cgemm_tf32x3(bem_ctx* ctx, int M, int N, int K, const void* A, int64_t lda, const void* B,
                     int64_t ldb, int b_rowmajor, void* C, int64_t ldc, int c_colmajor);

/* ---------------------------------------------------------- whole pipeline */

typedef struct bem_problem {
    /* mesh (host) */
    const double* verts; int nv; const int* tris; int nt;
    double ka;             /* k_ext = ka (unit equivalent radius) */
    double m_re, m_im;     /* relative refractive index; k_int = k_ext m, eta_int = 1/|m| */
    int quad_order;        /* 4, 7 or 13 */
    int single;            /* 1: k_hat = z, E = x / y (main.cpp:671-718) */
    int n_alpha, n_beta, n_gamma;
    int beta_sym, gamma_sym, gamma_mirror;
    int orient_i0, orient_i1;  /* orientation range [i0, i1), -1 = all */
    int ntheta;
    int precision;         /* bem_precision */
    double refine_tol;     /* <= 0: 1e-12 */
    int max_refine;        /* <= 0: 10 */
    unsigned asm_flags;
    /* Adaptive orientation stopping (main.cpp:477-636): orientations are solved
     * in batches of max(20, n/20) with the one factorisation; after each batch
     * from 40 orientations on, the scattering-cross-section proxy
     * sum_{t=3}^{ntheta-4} M11(t) sin(theta_t) / w_sum is compared with the
     * previous batch's; two consecutive relative changes below orient_tol stop
     * the loop and the average is rescaled to the full weight.  0 = off. */
    double orient_tol;
    /* Solver of the orientation columns: BEM_SOLVER_LU (the LU of Z, default)
     * or BEM_SOLVER_GMRES_AEXT (GMRES on Z with the LU of the exterior-only
     * A_ext as preconditioner, per column as the reference's
     * orientation-averaging functions do when given Z_ext_lu,
     * bem_core.py:1703-1709; `precision` then applies to A_ext's LU).
     * gmres_tol <= 0: 1e-5; gmres_restart <= 0: min(200, 2N);
     * gmres_maxiter <= 0: 200 (solve_gmres_aext's defaults). */
    int solver;
    double gmres_tol;
    int gmres_restart;
    int gmres_maxiter;
} bem_problem;

#define BEM_SOLVER_LU 0
#define BEM_SOLVER_GMRES_AEXT 1

typedef struct bem_result {
    double* mueller;       /* caller buffer, 16 * ntheta doubles */
    double t_assembly_s, t_solve_s, t_farfield_s, t_total_s;
    int N, n_orient;
    bem_solve_stats stats;
    /* optional per-orientation stream (the .per_orient file of main.cpp:640-653):
     * per_orient_mueller[o*16*ntheta + i*ntheta + t] = M_o (amplitude_to_mueller,
     * no weight, no 1/|k|^2) and per_orient_weight[o], for the n_computed first
     * orientations; caller buffers sized for n_orient orientations, or NULL. */
    double* per_orient_mueller;
    double* per_orient_weight;
    int n_computed;        /* orientations solved (< n_orient after an adaptive stop) */
    double t_setup_s;      /* geometry upload, orientations and device buffers */
    double t_release_s;    /* freeing the device buffers */
    bem_gmres_stats gmres; /* BEM_SOLVER_GMRES_AEXT: over all batches */
} bem_result;

/* The dense branch of main.cpp (:660-854) end to end on the device: assemble,
 * factor, solve every orientation x polarisation at once, far field, Mueller. */
int bem_dense_run(bem_ctx* ctx, const bem_problem* p, bem_result* r);

/* Adjoint gradient of an orientation-averaged M11 misfit,
 *   loss = sum_t wt[t] (M11(theta_t) - target[t])^2   (wt NULL: 1),
 * with respect to the relative refractive index (grad[0] = dloss/dRe m,
 * grad[1] = dloss/dIm m), for the problem p (mesh, ka, m, orientations,
 * ntheta; its precision is ignored: FP64 forward and adjoint solves).
 * mueller (optional, 16 ntheta) receives the forward Mueller matrix.  The
 * reference has no gradient code; the result is checked against central
 * differences of the forward path. */
int bem_adjoint_grad(bem_ctx* ctx, const bem_problem* p, const double* target, const double* wt,
                     double* loss, double* grad, double* mueller);
/* The same misfit's gradient with respect to the vertex coordinates of the
 * mesh (grad_verts: 3 nv doubles, x y z per vertex): the adjoint vectors of
 * one forward and one adjoint solve, contracted per coordinate with the
 * central differences (h = 1e-6) of the operator, the right-hand sides and
 * the far field assembled on the moved geometry (no re-solve). */
int bem_adjoint_grad_vertices(bem_ctx* ctx, const bem_problem* p, const double* target, const double* wt,
                              double* loss, double* grad_verts, double* mueller);

/* Batched particles (many small scatterers, e.g. the seeded hex-prism sets
 * that cluster_bem.py farms out one process per particle): the dense pipeline
 * for problems[0..count) on this context, results[i] for each.  FP64
 * particles of one system size (LU solver, no adaptive stopping, no
 * per-orientation output, full orientation set) run as a bucket: their
 * operators assembled into one batch, one batched LU and one batched solve
 * (each launch covering every particle of the size; option batch_buckets),
 * with the LU's block / panel widths from the autotuner (lu_autotune); the
 * bucket's phase times are shared equally by its particles' results.  Other
 * particles run one at a time as bem_dense_run.  statuses[i] (optional) gets
 * each particle's status and a failure does not stop the batch.  Returns
 * BEM_OK or the first particle's failure. */
int bem_batch_run(bem_ctx* ctx, const bem_problem* problems, int count, bem_result* results,
                  int* statuses);

#ifdef __cplusplus
}
#endif
#endif /* BEM_DENSE_H */
