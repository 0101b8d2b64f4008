// Internal declarations shared by the libbemdense translation units.
#pragma once

#include <cuda_runtime.h>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "bem_dense.h"

namespace bem {

// ---------------------------------------------------------------- errors
struct Error {
    int status;
    std::string msg;
};

// Records a failure on the context and returns its status.
int fail(bem_ctx* ctx, int status, const char* fmt, ...);

// Host <-> device copies in the context's stream order (its stream may be a
// non-blocking one, which the legacy default stream of cudaMemcpy does not
// wait for): h2d stages the host data before it returns and precedes the
// kernels launched after it; d2h waits for the stream, so the data is on the
// host when it returns.
int h2d(bem_ctx* ctx, void* dst, const void* src, size_t bytes);
int d2h(bem_ctx* ctx, void* dst, const void* src, size_t bytes);

#define BEM_TRY_CUDA(ctx, call)                                                         \
    do {                                                                                \
        cudaError_t e__ = (call);                                                       \
        if (e__ != cudaSuccess) {                                                       \
            return ::bem::fail((ctx), e__ == cudaErrorMemoryAllocation ? BEM_ERR_OOM    \
                                                                       : BEM_ERR_CUDA,  \
                               "%s:%d %s: %s", __FILE__, __LINE__, #call,              \
                               cudaGetErrorString(e__));                                \
        }                                                                               \
    } while (0)

#define BEM_TRY(call)              \
    do {                           \
        int s__ = (call);          \
        if (s__ != BEM_OK) return s__; \
    } while (0)

// Launch check: records the launch and reports launch-configuration errors.
#define BEM_LAUNCHED(ctx)                                                              \
    do {                                                                               \
        (ctx)->launches++;                                                             \
        cudaError_t e__ = cudaGetLastError();                                          \
        if (e__ != cudaSuccess)                                                        \
            return ::bem::fail((ctx), BEM_ERR_CUDA, "%s:%d launch: %s", __FILE__,     \
                               __LINE__, cudaGetErrorString(e__));                     \
    } while (0)

// ------------------------------------------------------------ host geometry
struct V3 {
    double x, y, z;
};

struct HostMesh {
    std::vector<V3> verts;
    std::vector<int> tris;  // 3 per triangle
    int nv() const { return (int)verts.size(); }
    int nt() const { return (int)tris.size() / 3; }
};

struct HostRWG {
    int N = 0;
    std::vector<int> tri_p, tri_m;
    std::vector<int> vfree_p, vfree_m;  // vertex index of the free vertices
    std::vector<V3> free_p, free_m;
    std::vector<double> length, area_p, area_m;
    std::vector<int> edge_lo, edge_hi;  // vertex indices of the edge (empty: basis given by the caller)
};

struct Quad {
    int n = 0;
    double l1[25], l2[25], w[25];
};

bool host_mesh_from(const double* verts, int nv, const int* tris, int nt, HostMesh* m);
HostMesh make_icosphere(double radius, int refinements);
HostMesh make_hex_prism(double aspect_ratio, int refinements);
HostMesh subdivide_flat(const HostMesh& m);
HostRWG build_rwg(const HostMesh& m);
// Free vertices, edge lengths and areas of a mesh-built basis after the
// vertices moved (same formulas as build_rwg).
void rwg_refresh(const HostMesh& m, HostRWG& r);
bool quadrature(int order, Quad* q);  // false: unsupported order
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w);
void orientations(int na, int nb, int ng, int bsym, int gsym, bool mirror, bool sort,
                  std::vector<double>& RT, std::vector<double>& w);
double tri_area(const HostMesh& m, int t);

// ---------------------------------------------------------- device geometry
// Quadrature data of every (RWG, half): index h*N + n, point q at
// ((h*N + n)*Nq + q).  Structure of arrays, all FP64.
struct DevHalf {
    double *px, *py, *pz;   // quadrature points
    double *fx, *fy, *fz;   // basis values sign*(l/2A)(r - r_free)
    double *cx, *cy, *cz;   // f x r (for the K triple product)
    double* jw;             // A * w_q
    double* div;            // (2N) sign*l/A
    int* tri;               // (2N) triangle of the half
};

// Same-triangle (singular) bookkeeping.  Every unordered pair {m, n} of RWG
// functions that share a triangle gets one slot; item_* lists the
// (triangle, test half, source half) combinations feeding it, CSR by slot.
struct DevSingular {
    int npairs = 0, nitems = 0;
    int* pair_mn;       // (2*npairs) m <= n
    int* item_ptr;      // (npairs+1)
    int* item;          // (nitems*3): triangle, test half index h*N+m, source half h*N+n
    double* P;          // (nt*Nq) Graglia potential at the triangle's points
    double* V;          // (nt*Nq*3) vector potential at the triangle's points
    double* tv;         // (nt*9) triangle vertices
};

// Device-memory cache for the large per-factorisation blocks (FP32 factors,
// int8 digit planes of Z).  While enabled for a device (the
// "cache_factor_memory" option), blocks freed there are kept and handed to
// the next request of exactly the same size, so a loop of factorisations of
// one size allocates once.  Per device and process-wide, so a factorisation
// may outlive the context that made it.  Disabling frees the kept blocks; an
// allocation that fails frees them and retries once.
// owner: the context whose stream uses the block (cached blocks are handed
// back only to their owner, in its stream order; null: any, after a device
// synchronisation).  Contexts register as owners while they live.
void* devmem_alloc(int device, size_t bytes, const void* owner);  // nullptr when out of memory
void devmem_free(int device, void* p, size_t bytes, const void* owner);
void devmem_owner(const void* owner, bool alive);
void devmem_cache_enable(int device, bool on);
bool devmem_cache_enabled(int device);

// Triangle-pair assembly: per-triangle quadrature data relative to the
// centroid, and the RWGs in tiles of ASM_TILE ordered along a Morton curve of
// their triangles' centroids, so that the RWGs of a tile share triangles.
constexpr int ASM_TRI_MAX = 32;  // distinct triangles of one tile (2 halves x 16 RWGs at most)
struct DevTriAsm {
    double* c = nullptr;          // (nt, 3) centroids
    double* u = nullptr;          // (nt, Nq, 3) quadrature points minus the centroid
    double* jw = nullptr;         // (nt, Nq) area x weight
    double* pi = nullptr;         // (2N, 3) free vertex of half h*N+n minus its triangle's centroid
    int* tile_rwg = nullptr;      // (ntile, 16) RWG of each tile slot, -1 past N
    int* pos = nullptr;           // (N) slot of each RWG: tile = pos / 16
    int* tile_tri = nullptr;      // (ntile, ASM_TRI_MAX) distinct triangles of the tile, -1 padded
    int* tile_ntri = nullptr;     // (ntile)
    unsigned char* tile_ent = nullptr;  // (ntile, ASM_TRI_MAX, 3): slot * 2 + half on the triangle, 0xff none
    int* tri_half = nullptr;      // (nt, 3) RWG halves h*N+n on each triangle, -1 padded
    unsigned char* tile_flag = nullptr; // (ntile) scratch: tiles to recompute
    unsigned char* rwg_rec = nullptr;   // (N) scratch: RWGs whose tile is recomputed
    int ntile = 0;
};

}  // namespace bem

// Per-kernel-class timing (CUDA events around the launches of one class on
// the context's stream), enabled by bem_ctx_profile.
enum ProfClass {
    PROF_LU_UPDATE = 0,    // trailing update GEMM of the factorisation
    PROF_SOLVE_UPDATE = 1, // block updates of the triangular solves
    PROF_RESIDUAL = 2,     // FP64 refinement residual B - Z X
    PROF_PANEL = 3,        // panel factorisation kernels
    PROF_ASSEMBLY = 4,     // PMCHWT assembly kernel
    PROF_FARFIELD = 5,     // far-field / Mueller kernel
    PROF_VERIFY = 6,       // FP64 residual of the columns checked after the refinement
    PROF_TRSM = 7,         // triangular solves with a 256-row diagonal block (factorisations and solves)
    PROF_PIVOT = 8,        // row interchanges and permutations
    PROF_PANEL_UPDATE = 9, // updates inside a block column (sub-panel GEMMs; L21 of the L D L^T blocks)
    PROF_NCLASS = 10
};

struct ProfPending {
    int cls;
    cudaEvent_t a, b;
    double flops, bytes;
};

struct bem_ctx {
    int device = 0;
    bool use_tc = true;  // FP32 updates on the tensor cores (else CUDA cores)
    float* tc_buf = nullptr;  // packed hi/lo operands of the tensor-core GEMM
    size_t tc_bytes = 0;
    bool tc_attr = false;
    int ff_kernel = 0;           // far field: 0 by triangles (shared phases), 1 per RWG-half point
    int asm_kernel = 0;          // assembly: 0 triangle-pair moments (Morton tiles), 1 per RWG pair
    int tc_group_m = 16;         // row tiles per raster group of the persistent tensor-core GEMM
    bool tc_persistent = true;  // persistent tensor-core GEMM (else one CTA per tile)
    bool tc_pair = true;        // FP16-part GEMM on CTA pairs (cta_group::2, 256-row tiles)
    bool tc_pair_attr = false;
    bool dmma_3m = true;        // complex FP64 GEMMs as three real products (Gauss) instead of four
    bool solve_inv = true;      // L D L^T solves: diagonal blocks by products with their stored inverses
    bool ldlt_cluster = true;   // L D L^T factor: diagonal blocks on an 8-CTA cluster (else one CTA)
    bool lu_u12_slabs = true;  // FP64 LU: U12 by 64-row slabs with GEMM updates between them
    int tc_split = 1;           // FP32 operand split: 1 = 3xFP16 with power-of-two row / column scales, 0 = 3xTF32
    int sym_mode = 1;            // FP32 factorisation of symmetric-structured Z as L D L^T (0: always LU)
    int oz_digits = 7;           // int8 digits of the Ozaki residual (0: FP64 DMMA residual)
    int oz_xdigits = 2;          // digits the refinement keeps of its first iterate and of its corrections (0: all)
    void* oz_buf = nullptr;      // digit planes of X for the residual
    size_t oz_bytes = 0;
    bool oz_attr = false;
    int gmres_digits = 0;        // GMRES products with Z: 0 FP64 DMMA GEMM, 2..8 int8 Ozaki digits
    bool batch_buckets = true;   // bem_batch_run: FP64 particles of one size batched (else one at a time)
    bool lu_autotune = true;     // batched LU shape from the autotuner (else NB 256, W 16)
    bool panel_clusters = true;  // LU sub-panels that fit one thread-block cluster run on it (cluster
                                 // barrier per column) instead of the cooperative grid
    int grad_method = 0;         // adjoint gradients: 0 contraction kernels (grad_geom.cu), 1 central
                                 // differences of reassembled operators
    int verify_cols = 64;        // refinement: columns whose error is measured with an FP64 residual
                                 // at convergence (0: none, -1: all)
    int factor_sb = 4;           // L D L^T: 256-column blocks per trailing update (1..4)
    int solve_sb = 4;            // L D L^T solves: 256-row blocks per update (1..4)
    int oz_pace_epoch = 32;      // int8 residual: K slabs per pacing epoch (0: no pacing)
    int oz_pace_lead = 2;        // epochs of lead over the grid average before a CTA waits
    bool prof = false;
    std::vector<ProfPending> prof_pending;
    std::vector<cudaEvent_t> prof_pool;
    int64_t prof_launches[PROF_NCLASS] = {0};
    double prof_ms[PROF_NCLASS] = {0}, prof_flops[PROF_NCLASS] = {0}, prof_bytes[PROF_NCLASS] = {0};
    cudaEvent_t prof_begin(int cls);
    void prof_end(int cls, cudaEvent_t a, double flops, double bytes);
    int prof_collect();
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    int sm_count = 148;
    int64_t launches = 0;
    std::string last_error;
    // bounded-wait status word for device-side barriers (0 = ok)
    int* d_status = nullptr;
    // reusable device workspace
    void* ws = nullptr;
    size_t ws_bytes = 0;
    int ensure_ws(size_t bytes);
};

struct bem_geom {
    bem_ctx* ctx = nullptr;  // creating context (not used after bem_geom_free starts)
    int device = 0;
    int N = 0, Nq = 0, nv = 0, nt = 0, quad_order = 7;
    bem::HostMesh mesh;
    bem::HostRWG rwg;
    bem::Quad quad;
    bem::DevHalf half{};
    bem::DevSingular sing{};
    double* sing_coef = nullptr;  // (2N) sign*l/(2A) per half
    double* sing_free = nullptr;  // (3*2N) free vertex per half, x | y | z blocks
    bem::DevTriAsm tri{};         // triangle-pair assembly data (Morton-ordered tiles)
    void* dmem = nullptr;  // one allocation backing every device array (devmem_alloc)
    size_t dmem_bytes = 0;
};

namespace bem {
// assembly.cu
// rwg_mask (device, optional): one flag per RWG; only the tiles holding a
// flagged RWG in their rows or columns are written (every entry of a flagged
// RWG among them; the other tiles keep their values, and entries recomputed
// without a flagged RWG come out bitwise as before).
int assemble_dev(bem_ctx* ctx, const bem_geom* g, double ke_re, double ke_im, double ki_re,
                 double ki_im, double eta_e, double eta_i, unsigned flags, int mode,
                 void* Z, int64_t ldz, void* L, void* K, const unsigned char* rwg_mask = nullptr);
constexpr int ASM_TILE = 16;  // RWGs per assembly band
int geom_upload(bem_ctx* ctx, bem_geom* g);
// Moves the vertices of a geometry made by bem_geom_create (nv x 3 doubles)
// and refreshes every position-dependent device array in place, in the
// context's stream order: same topology, RWG order, tiles and allocation.
// Right-hand sides and far field equal a new geometry's; the operator does to
// rounding (the kept tiles fix which orientation of a symmetric pair is computed).
int geom_set_vertices(bem_ctx* ctx, bem_geom* g, const double* verts);
// Batched FP64 LU of `batch` equally sized row-major matrices A + i sA
// (pivots d_ipiv + i n, info d_info + i): every step of the blocked
// factorisation is one launch for the whole batch (the panel kernel's CTAs
// of all matrices meet at one grid barrier).  NB: block columns per trailing
// update, W: panel width (<= 32); the shapes the autotuner chooses from.
struct LuShape {
    int NB = 256, W = 16;
};
int getrf_batched(bem_ctx* ctx, double2* A, int64_t lda, int64_t sA, int n, int batch, int* d_ipiv, int* d_info,
                  LuShape shape);
// The batched LU's shape for (n, batch), chosen by timing the candidates
// once on test matrices of order n and kept for the process.
int tune_lu_shape(bem_ctx* ctx, int n, int batch, LuShape* out);
// X_i = (P_i^T L_i U_i)^-1 B_i for the batch (perm d_perm + i n).
int getrs_batched(bem_ctx* ctx, const double2* LU, int64_t lda, int64_t sA, int n, int batch, const int* d_perm,
                  const double2* B, int64_t ldb, int64_t sB, double2* X, int64_t ldx, int64_t sX, int nrhs,
                  int NB = 256);

void pivots_to_perm(const std::vector<int>& ipiv, std::vector<int>& perm);
// grad_geom.cu: the adjoint contractions of the shape gradient.  X, Lam:
// forward and adjoint solutions (column-major 2N x ncols); RT_dev, hp_dev,
// rh_dev: the orientations and the far-field adjoint weights h and rhat x h
// per (column, angle, component) on the device.  grad_v (host, 3 nv, may be
// null) receives dloss/dv; dpsi_dk (host, 4 doubles) the complex
// contractions sum S . d(Z D)/dRe k_int and sum S . d(Z D)/dIm k_int,
// dpsi_deta (2 doubles) sum S . d(Z D)/deta_int.
int adjoint_geometry(bem_ctx* ctx, const bem_geom* g, std::complex<double> kext, std::complex<double> kint,
                     double eta_e, double eta_i, unsigned flags, const void* X, const void* Lam, int ncols,
                     const double* RT_dev, int n_orient, const void* hp_dev, const void* rh_dev, int ntheta,
                     double* grad_v, double* dpsi_dk, double* dpsi_deta);
// rhs / farfield
int rhs_dev(bem_ctx* ctx, const bem_geom* g, double k_re, double k_im, double eta,
            const double* RT_host, const double* E0_host, const double* khat_host, int n_orient,
            void* B, int64_t ldb);
int farfield_dev(bem_ctx* ctx, const bem_geom* g, const void* X, int64_t ldx, int n_calls_x,
                 const double* coeffJ_host, const double* coeffM_host, const double* rhat_host,
                 int n_orient, int ndir, double k_re, double k_im, double eta, double* Fv_host);
int mueller_dev(bem_ctx* ctx, const bem_geom* g, const void* X, int64_t ldx, const double* RT,
                const double* w, int n_orient, double k_re, double k_im, double eta,
                int ntheta, int gamma_mirror, double* M_avg, double* M_orient_dev,
                double* Fv_host = nullptr);
}  // namespace bem
