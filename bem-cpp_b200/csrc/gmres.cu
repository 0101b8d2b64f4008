// GMRES(m) on the dense PMCHWT matrix, many right-hand sides at once, with
// the preconditioners of the reference's iterative dense solves:
//   solve_gmres_aext  bem_core.py:1093-1123  (A_ext LU, restart min(200, n))
//   solve_gmres       bem_core.py:1126-1183  ('block_diag', 'diag', None)
//   build_aext_preconditioner bem_core.py:1071-1090 (assembly.cu mode 3)
// Both call scipy.sparse.linalg.gmres (SciPy 1.18.1,
// scipy/sparse/linalg/_isolve/iterative.py), whose algorithm is restated here
// column by column: left preconditioning, modified Gram-Schmidt Arnoldi,
// complex Givens rotations (LAPACK zlartg convention), the inner loop ends
// when the preconditioned residual estimate falls below ptol (tolerance
// control of gh-8400), each restart cycle recomputes b - Z x in FP64 and the
// solve ends when ||b - Z x||_2 <= tol ||b||_2 or after maxiter cycles.
//
// B200 layout: the columns of a chunk share every product with Z (one GEMM
// over the columns still in their inner loop), the Gram-Schmidt sweep of a
// step is one kernel with one CTA per column, and the small Hessenberg /
// Givens state (restart^2 numbers per column) lives on the host.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>

#include "bem_internal.h"
#include "lu_internal.h"
#include "ozaki.h"

struct bem_precond {
    int kind = BEM_PRECOND_NONE;
    int n = 0;
    int device = 0;
    bem_lu* lu = nullptr;              // BEM_PRECOND_LU (caller's)
    bem_lu* blk[2] = {nullptr, nullptr};  // BEM_PRECOND_BLOCK_DIAG (owned)
    double2* blk_z[2] = {nullptr, nullptr};  // FP64 copies of Z11, Z22 (owned)
    double2* dinv = nullptr;           // BEM_PRECOND_DIAG: 1 / diag(Z) (owned)
};

namespace bem {
namespace {

using cplx = std::complex<double>;

unsigned nblk(int64_t tot) { return (unsigned)((tot + 255) / 256); }

// Z11 / Z22 copy: dst[i*ld + j] = Z[(r0+i)*ldz + r0+j], i, j < m.
__global__ void copy_block_kernel(const double2* __restrict__ Z, int64_t ldz, int r0, int m,
                                  double2* __restrict__ dst) {
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)m * m) return;
    const int i = (int)(t / m), j = (int)(t % m);
    dst[t] = Z[(int64_t)(r0 + i) * ldz + r0 + j];
}

__global__ void inv_diag_kernel(const double2* __restrict__ Z, int64_t ldz, int n, double2* __restrict__ d,
                                int* __restrict__ zero) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double2 z = Z[(int64_t)i * ldz + i];
    double a = z.x * z.x + z.y * z.y;
    if (a == 0.0) {
        atomicExch(zero, 1);
        d[i] = make_double2(0.0, 0.0);
        return;
    }
    // the reference divides x / d (bem_core.py:1160-1162); 1/d rounded once
    d[i] = make_double2(z.x / a, -z.y / a);
}

// Y[:, p] = D^-1 X[:, p]
__global__ void apply_diag_kernel(const double2* __restrict__ dinv, const double2* __restrict__ X, int64_t ldx,
                                  double2* __restrict__ Y, int64_t ldy, int n, int nc) {
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)n * nc) return;
    const int r = (int)(t % n), c = (int)(t / n);
    double2 a = dinv[r], x = X[(int64_t)c * ldx + r];
    Y[(int64_t)c * ldy + r] = make_double2(a.x * x.x - a.y * x.y, a.x * x.y + a.y * x.x);
}

// P[:, p] = s * src[:, idx[p]] (columns of the slot-layout block src, ld n)
__global__ void gather_kernel(const double2* __restrict__ src, int64_t lds, const int* __restrict__ idx,
                              double s, double2* __restrict__ P, int n, int na) {
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)n * na) return;
    const int r = (int)(t % n), p = (int)(t / n);
    double2 v = src[(int64_t)idx[p] * lds + r];
    P[(int64_t)p * n + r] = make_double2(s * v.x, s * v.y);
}

// Per packed column: out[p] = ||X[:, p]||_2, then (when V0 given)
// V0[:, idx[p]] = X[:, p] * (1 / out[p]) -- the start vector of a cycle.
__global__ void norm_kernel(const double2* __restrict__ X, int n, double* __restrict__ out,
                            double2* __restrict__ V0, const int* __restrict__ idx) {
    __shared__ double red[32];
    __shared__ double s_tot;
    const double2* x = X + (int64_t)blockIdx.x * n;
    double acc = 0.0;
    for (int r = threadIdx.x; r < n; r += blockDim.x) acc += x[r].x * x[r].x + x[r].y * x[r].y;
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) s_tot = sqrt(v);
    }
    __syncthreads();
    const double nrm = s_tot;
    if (threadIdx.x == 0) out[blockIdx.x] = nrm;
    if (!V0) return;
    const double inv = nrm > 0.0 ? 1.0 / nrm : 0.0;
    double2* v = V0 + (int64_t)idx[blockIdx.x] * n;
    for (int r = threadIdx.x; r < n; r += blockDim.x) v[r] = make_double2(x[r].x * inv, x[r].y * inv);
}

// Sum over the CTA of (re, im); every thread gets the total.
__device__ double2 block_sum2(double re, double im, double2* red) {
    for (int o = 16; o; o >>= 1) {
        re += __shfl_xor_sync(0xffffffffu, re, o);
        im += __shfl_xor_sync(0xffffffffu, im, o);
    }
    const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    __syncthreads();  // red reused across calls
    if ((threadIdx.x & 31) == 0) red[w] = make_double2(re, im);
    __syncthreads();
    double2 t = make_double2(0.0, 0.0);
    for (int i = 0; i < nw; i++) t.x += red[i].x, t.y += red[i].y;
    return t;
}

// One Arnoldi step of modified Gram-Schmidt for packed column p (slot
// idx[p]): h0 = ||w||; for k <= col: h_k = <v_k, w>, w -= h_k v_k; h1 = ||w||;
// v_{col+1} = w (times 1/h1 unless h1 <= eps h0).  H[p*(col+3) + k] = h_k,
// [col+1] = h1 (0 on breakdown), [col+2] = h0.  V: slot-layout blocks.
__global__ void __launch_bounds__(512) mgs_kernel(double2* __restrict__ W, int n, double2* const* __restrict__ V,
                                                  const int* __restrict__ idx, int col, double2* __restrict__ H) {
    __shared__ double2 red[16];
    const int p = blockIdx.x;
    const int64_t off = (int64_t)idx[p] * n;
    double2* w = W + (int64_t)p * n;
    double2* hout = H + (int64_t)p * (col + 3);
    double a = 0.0;
    for (int r = threadIdx.x; r < n; r += blockDim.x) a += w[r].x * w[r].x + w[r].y * w[r].y;
    const double h0 = sqrt(block_sum2(a, 0.0, red).x);
    for (int k = 0; k <= col; k++) {
        const double2* v = V[k] + off;
        double re = 0.0, im = 0.0;
        for (int r = threadIdx.x; r < n; r += blockDim.x) {
            const double2 x = v[r], y = w[r];
            re += x.x * y.x + x.y * y.y;  // conj(v) w
            im += x.x * y.y - x.y * y.x;
        }
        const double2 h = block_sum2(re, im, red);
        for (int r = threadIdx.x; r < n; r += blockDim.x) {
            const double2 x = v[r];
            double2 y = w[r];
            y.x -= h.x * x.x - h.y * x.y;
            y.y -= h.x * x.y + h.y * x.x;
            w[r] = y;
        }
        if (threadIdx.x == 0) hout[k] = h;
    }
    __syncthreads();
    a = 0.0;
    for (int r = threadIdx.x; r < n; r += blockDim.x) a += w[r].x * w[r].x + w[r].y * w[r].y;
    const double h1 = sqrt(block_sum2(a, 0.0, red).x);
    const bool breakdown = h1 <= 2.220446049250313e-16 * h0;
    const double inv = breakdown ? 1.0 : 1.0 / h1;
    double2* vn = V[col + 1] + off;
    for (int r = threadIdx.x; r < n; r += blockDim.x) vn[r] = make_double2(w[r].x * inv, w[r].y * inv);
    if (threadIdx.x == 0) {
        hout[col + 1] = make_double2(breakdown ? 0.0 : h1, 0.0);
        hout[col + 2] = make_double2(h0, 0.0);
    }
}

// X[:, xcol[p]] += sum_{k < kc[p]} Y[p*ystride + k] V_k[:, idx[p]]
__global__ void update_x_kernel(double2* __restrict__ X, int64_t ldx, const int* __restrict__ xcol,
                                double2* const* __restrict__ V, const int* __restrict__ idx,
                                const double2* __restrict__ Y, int ystride, const int* __restrict__ kc, int n,
                                int na) {
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)n * na) return;
    const int r = (int)(t % n), p = (int)(t / n);
    const int64_t off = (int64_t)idx[p] * n + r;
    const double2* y = Y + (int64_t)p * ystride;
    double2 acc = make_double2(0.0, 0.0);
    for (int k = 0; k < kc[p]; k++) {
        const double2 v = V[k][off], c = y[k];
        acc.x += c.x * v.x - c.y * v.y;
        acc.y += c.x * v.y + c.y * v.x;
    }
    double2* x = &X[(int64_t)xcol[p] * ldx + r];
    x->x += acc.x;
    x->y += acc.y;
}

__global__ void zero_cols_kernel(double2* __restrict__ X, int64_t ldx, int c0, int n, int nc) {
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)n * nc) return;
    X[(int64_t)(c0 + t / n) * ldx + t % n] = make_double2(0.0, 0.0);
}

// LAPACK zlartg: c real, s complex with [c s; -conj(s) c] [f; g] = [r; 0].
void zlartg(cplx f, cplx g, double* c, cplx* s, cplx* r) {
    if (g == 0.0) {
        *c = 1.0, *s = 0.0, *r = f;
        return;
    }
    if (f == 0.0) {
        const double ag = std::abs(g);
        *c = 0.0, *s = std::conj(g) / ag, *r = ag;
        return;
    }
    const double af = std::abs(f), ag = std::abs(g), d = std::hypot(af, ag);
    const cplx ph = f / af;
    *c = af / d;
    *s = ph * std::conj(g) / d;
    *r = ph * d;
}

struct Col {
    double bnrm2 = 0, atol = 0, ptol = 0, ptol_max_factor = 1, presid = 0, rnorm = 0;
    int cycles = 0, inner = 0, info = 0;
    bool done = false, breakdown = false, in_loop = false;
    int kend = 0;  // Krylov vectors used in this cycle
    std::vector<cplx> H, S, gs;
    std::vector<double> gc;
};

}  // namespace

// M^-1 X -> Y for nc packed columns (ld n); X and Y distinct.
static int precond_apply(bem_ctx* ctx, bem_precond* M, const double2* X, double2* Y, int nc) {
    const int n = M->n;
    const int64_t tot = (int64_t)n * nc;
    switch (M->kind) {
        case BEM_PRECOND_NONE:
            BEM_TRY_CUDA(ctx, cudaMemcpyAsync(Y, X, tot * sizeof(double2), cudaMemcpyDeviceToDevice, ctx->stream));
            return BEM_OK;
        case BEM_PRECOND_DIAG:
            apply_diag_kernel<<<nblk(tot), 256, 0, ctx->stream>>>(M->dinv, X, n, Y, n, n, nc);
            BEM_LAUNCHED(ctx);
            return BEM_OK;
        case BEM_PRECOND_BLOCK_DIAG: {
            const int h = n / 2;
            BEM_TRY(lu_apply(ctx, M->blk[0], X, n, Y, n, nc));
            return lu_apply(ctx, M->blk[1], X + h, n, Y + h, n, nc);
        }
        case BEM_PRECOND_LU:
            return lu_apply(ctx, M->lu, X, n, Y, n, nc);
    }
    return fail(ctx, BEM_ERR_INVALID, "unknown preconditioner kind %d", M->kind);
}

// R -= Z P for nc packed columns (ld n): the int8 Ozaki product when digit
// planes exist, else the FP64 tensor-core (DMMA) complex GEMM.
static int z_sub(bem_ctx* ctx, const double2* Z, int64_t ldz, int n, const OzakiZ* oz, const double2* P,
                 double2* R, int nc) {
    if (oz && oz->A) return ozaki_residual(ctx, oz, P, n, R, n, nc);
    return cgemm<double>(ctx, n, nc, n, Z, ldz, P, n, true, R, n, true, make_double2(-1, 0), make_double2(1, 0),
                         PROF_RESIDUAL);
}

static int sync_status(bem_ctx* ctx) {
    int h = 0;
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(&h, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    BEM_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (h != 0) return fail(ctx, h, "device-side wait in a tensor-core kernel of GMRES gave up");
    return BEM_OK;
}

namespace {
struct Bufs {
    std::vector<void*> all;
    ~Bufs() {
        for (void* p : all) cudaFree(p);
    }
    void* get(size_t bytes) {
        void* p = nullptr;
        if (cudaMalloc(&p, bytes) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        all.push_back(p);
        return p;
    }
};
}  // namespace

static int gmres_run(bem_ctx* ctx, const double2* Z, int n, int64_t ldz, bem_precond* M, const double2* B,
                     int64_t ldb, double2* X, int64_t ldx, int nrhs, int restart, double tol, int maxiter,
                     int* iters_out, int* info_out, bem_gmres_stats* st) {
    auto t0 = std::chrono::steady_clock::now();
    bem_gmres_stats stats;
    std::memset(&stats, 0, sizeof stats);
    stats.converged = 1;
    restart = std::min(restart, n);
    const int m = restart;
    // Z digit planes for the products (bem_ctx_set_option "gmres_digits")
    OzakiZ oz;
    struct OzGuard {
        OzakiZ* o;
        ~OzGuard() { ozaki_free(o); }
    } ozg{&oz};
    if (ctx->gmres_digits > 0 && ozaki_prepare_z(ctx, &oz, Z, ldz, n, ctx->gmres_digits) != BEM_OK)
        ozaki_free(&oz);
    // chunk width from the free memory: m + 1 basis blocks + 3 packed blocks
    // + the preconditioner's FP32 workspace per column
    size_t fmem = 0, tmem = 0;
    BEM_TRY_CUDA(ctx, cudaMemGetInfo(&fmem, &tmem));
    const size_t col_bytes = (size_t)n * 16;
    const size_t per_col = col_bytes * (std::min(m, 40) + 1 + 3) + (size_t)n * 40;
    int nbw = (int)std::max<size_t>(1, std::min<size_t>(nrhs, (size_t)(0.6 * fmem) / per_col));
    Bufs bufs;
    double2* P = (double2*)bufs.get(col_bytes * nbw);
    double2* T = (double2*)bufs.get(col_bytes * nbw);
    double2* W = (double2*)bufs.get(col_bytes * nbw);
    double* dnorm = (double*)bufs.get(sizeof(double) * nbw);
    int* didx = (int*)bufs.get(sizeof(int) * 3 * nbw);
    double2* dH = (double2*)bufs.get(sizeof(double2) * (size_t)nbw * (m + 3));
    double2* dY = (double2*)bufs.get(sizeof(double2) * (size_t)nbw * m);
    double2** dV = (double2**)bufs.get(sizeof(double2*) * (m + 1));
    if (!P || !T || !W || !dnorm || !didx || !dH || !dY || !dV)
        return fail(ctx, BEM_ERR_OOM, "GMRES work buffers (%d columns of %d)", nbw, n);
    std::vector<double2*> V;  // basis blocks, allocated on first use
    auto basis = [&](int k) -> int {
        while ((int)V.size() <= k) {
            double2* b = (double2*)bufs.get(col_bytes * nbw);
            if (!b)
                return fail(ctx, BEM_ERR_OOM, "GMRES Krylov basis: %d vectors of %d x %d (lower restart)",
                            (int)V.size() + 1, n, nbw);
            V.push_back(b);
            BEM_TRY_CUDA(ctx, cudaMemcpyAsync(dV, V.data(), V.size() * sizeof(double2*), cudaMemcpyHostToDevice,
                                              ctx->stream));
        }
        return BEM_OK;
    };
    BEM_TRY(basis(1));
    std::vector<int> hidx(3 * nbw);
    std::vector<double> hnorm(nbw);
    std::vector<double2> hH((size_t)nbw * (m + 3)), hY((size_t)nbw * m);
    BEM_TRY_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream));
    const double eps = 2.220446049250313e-16;

    for (int c0 = 0; c0 < nrhs; c0 += nbw) {
        const int nc = std::min(nbw, nrhs - c0);
        std::vector<Col> cols(nc);
        zero_cols_kernel<<<nblk((int64_t)n * nc), 256, 0, ctx->stream>>>(X, ldx, c0, n, nc);
        BEM_LAUNCHED(ctx);
        // ||b||; T = b (the first residual, x0 = 0)
        for (int j = 0; j < nc; j++) hidx[j] = c0 + j;
        BEM_TRY_CUDA(ctx, cudaMemcpyAsync(didx, hidx.data(), nc * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
        gather_kernel<<<nblk((int64_t)n * nc), 256, 0, ctx->stream>>>(B, ldb, didx, 1.0, T, n, nc);
        BEM_LAUNCHED(ctx);
        norm_kernel<<<nc, 256, 0, ctx->stream>>>(T, n, dnorm, nullptr, nullptr);
        BEM_LAUNCHED(ctx);
        BEM_TRY_CUDA(ctx, cudaMemcpyAsync(hnorm.data(), dnorm, nc * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        BEM_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        // columns of the cycle (slot j in the chunk; T column = position in `cyc`)
        std::vector<int> cyc;
        for (int j = 0; j < nc; j++) {
            Col& c = cols[j];
            c.bnrm2 = hnorm[j];
            c.atol = tol * c.bnrm2;
            if (c.bnrm2 == 0.0 || c.bnrm2 < c.atol) {  // x = 0 (b = 0, or tol > 1)
                c.done = true;
                continue;
            }
            c.H.assign((size_t)m * (m + 1), 0.0);
            c.S.assign(m + 1, 0.0);
            c.gs.assign(m, 0.0);
            c.gc.assign(m, 0.0);
            cyc.push_back(j);
        }
        // compact T to the cycle's columns (zero-norm columns dropped)
        if ((int)cyc.size() != nc && !cyc.empty()) {
            for (size_t q = 0; q < cyc.size(); q++) hidx[q] = cyc[q];
            BEM_TRY_CUDA(ctx, cudaMemcpyAsync(didx, hidx.data(), cyc.size() * sizeof(int), cudaMemcpyHostToDevice,
                                              ctx->stream));
            gather_kernel<<<nblk((int64_t)n * cyc.size()), 256, 0, ctx->stream>>>(T, n, didx, 1.0, P, n,
                                                                                 (int)cyc.size());
            BEM_LAUNCHED(ctx);
            std::swap(P, T);
        }
        bool first = true;
        while (!cyc.empty()) {
            const int na0 = (int)cyc.size();
            // v0 = M^-1 r, S[0] = ||v0||, V_0 = v0 / S[0]
            BEM_TRY(precond_apply(ctx, M, T, W, na0));
            for (int q = 0; q < na0; q++) hidx[q] = cyc[q];
            BEM_TRY_CUDA(ctx, cudaMemcpyAsync(didx, hidx.data(), na0 * sizeof(int), cudaMemcpyHostToDevice,
                                              ctx->stream));
            norm_kernel<<<na0, 256, 0, ctx->stream>>>(W, n, dnorm, V[0], didx);
            BEM_LAUNCHED(ctx);
            BEM_TRY_CUDA(ctx, cudaMemcpyAsync(hnorm.data(), dnorm, na0 * sizeof(double), cudaMemcpyDeviceToHost,
                                              ctx->stream));
            BEM_TRY(sync_status(ctx));
            for (int q = 0; q < na0; q++) {
                Col& c = cols[cyc[q]];
                const double tmp = hnorm[q];
                if (first) c.ptol = tmp * std::min(c.ptol_max_factor, c.atol / c.bnrm2);  // Mb_nrm2 = ||M^-1 b||
                std::fill(c.S.begin(), c.S.end(), 0.0);
                c.S[0] = tmp;
                c.breakdown = false;
                c.in_loop = true;
                c.kend = 0;
            }
            first = false;
            // inner loop: all cycle columns step together until each leaves
            std::vector<int> act = cyc;
            for (int col = 0; col < m && !act.empty(); col++) {
                const int na = (int)act.size();
                BEM_TRY(basis(col + 1));
                for (int q = 0; q < na; q++) hidx[q] = act[q];
                BEM_TRY_CUDA(ctx, cudaMemcpyAsync(didx, hidx.data(), na * sizeof(int), cudaMemcpyHostToDevice,
                                                  ctx->stream));
                // T = Z v_col (P = -v_col, T = 0 - Z P); W = M^-1 T
                gather_kernel<<<nblk((int64_t)n * na), 256, 0, ctx->stream>>>(V[col], n, didx, -1.0, P, n, na);
                BEM_LAUNCHED(ctx);
                BEM_TRY_CUDA(ctx, cudaMemsetAsync(T, 0, col_bytes * na, ctx->stream));
                BEM_TRY(z_sub(ctx, Z, ldz, n, &oz, P, T, na));
                stats.matvecs++;
                BEM_TRY(precond_apply(ctx, M, T, W, na));
                mgs_kernel<<<na, 512, 0, ctx->stream>>>(W, n, dV, didx, col, dH);
                BEM_LAUNCHED(ctx);
                BEM_TRY_CUDA(ctx, cudaMemcpyAsync(hH.data(), dH, sizeof(double2) * (size_t)na * (col + 3),
                                                  cudaMemcpyDeviceToHost, ctx->stream));
                BEM_TRY(sync_status(ctx));
                std::vector<int> next;
                for (int q = 0; q < na; q++) {
                    Col& c = cols[act[q]];
                    cplx* h = &c.H[(size_t)col * (m + 1)];
                    const double2* hh = &hH[(size_t)q * (col + 3)];
                    for (int k = 0; k <= col + 1; k++) h[k] = cplx(hh[k].x, hh[k].y);
                    // the kernel stores h1 = 0 exactly when h1 <= eps h0 (breakdown)
                    c.breakdown = hh[col + 1].x == 0.0;
                    // previous rotations
                    for (int k = 0; k < col; k++) {
                        const double cc = c.gc[k];
                        const cplx ss = c.gs[k], n0 = h[k], n1 = h[k + 1];
                        h[k] = cc * n0 + ss * n1;
                        h[k + 1] = -std::conj(ss) * n0 + cc * n1;
                    }
                    double cc;
                    cplx ss, mag;
                    zlartg(h[col], h[col + 1], &cc, &ss, &mag);
                    c.gc[col] = cc, c.gs[col] = ss;
                    h[col] = mag, h[col + 1] = 0.0;
                    const cplx tmp = -std::conj(ss) * c.S[col];
                    c.S[col] = cc * c.S[col];
                    c.S[col + 1] = tmp;
                    c.presid = std::abs(tmp);
                    c.inner++;
                    c.kend = col + 1;
                    if (c.presid <= c.ptol || c.breakdown)
                        c.in_loop = false;
                    else
                        next.push_back(act[q]);
                }
                act.swap(next);
            }
            // y = H(0:k, 0:k)^-1 S(0:k); x += V y (per column, k = kend)
            const int na1 = (int)cyc.size();
            std::vector<int> kc(na1);
            for (int q = 0; q < na1; q++) {
                Col& c = cols[cyc[q]];
                const int col = c.kend - 1;
                auto Hc = [&](int i, int k) -> cplx& { return c.H[(size_t)i * (m + 1) + k]; };  // h[i, k]
                if (Hc(col, col) == 0.0) c.S[col] = 0.0;
                std::vector<cplx> y(c.S.begin(), c.S.begin() + col + 1);
                for (int k = col; k > 0; k--) {
                    if (y[k] != 0.0) {
                        y[k] /= Hc(k, k);
                        const cplx tmp = y[k];
                        for (int i = 0; i < k; i++) y[i] -= tmp * Hc(k, i);
                    }
                }
                if (y[0] != 0.0) y[0] /= Hc(0, 0);
                for (int k = 0; k <= col; k++) hY[(size_t)q * m + k] = make_double2(y[k].real(), y[k].imag());
                kc[q] = c.kend;
                hidx[q] = cyc[q];                 // slot
                hidx[nbw + q] = c0 + cyc[q];      // column of X
                hidx[2 * nbw + q] = c.kend;
            }
            BEM_TRY_CUDA(ctx, cudaMemcpyAsync(dY, hY.data(), sizeof(double2) * (size_t)na1 * m, cudaMemcpyHostToDevice,
                                              ctx->stream));
            BEM_TRY_CUDA(ctx, cudaMemcpyAsync(didx, hidx.data(), sizeof(int) * 3 * nbw, cudaMemcpyHostToDevice,
                                              ctx->stream));
            update_x_kernel<<<nblk((int64_t)n * na1), 256, 0, ctx->stream>>>(X, ldx, didx + nbw, dV, didx, dY, m,
                                                                           didx + 2 * nbw, n, na1);
            BEM_LAUNCHED(ctx);
            // r = b - Z x
            gather_kernel<<<nblk((int64_t)n * na1), 256, 0, ctx->stream>>>(B, ldb, didx + nbw, 1.0, T, n, na1);
            BEM_LAUNCHED(ctx);
            gather_kernel<<<nblk((int64_t)n * na1), 256, 0, ctx->stream>>>(X, ldx, didx + nbw, 1.0, P, n, na1);
            BEM_LAUNCHED(ctx);
            BEM_TRY(z_sub(ctx, Z, ldz, n, &oz, P, T, na1));
            stats.matvecs++;
            norm_kernel<<<na1, 256, 0, ctx->stream>>>(T, n, dnorm, nullptr, nullptr);
            BEM_LAUNCHED(ctx);
            BEM_TRY_CUDA(ctx, cudaMemcpyAsync(hnorm.data(), dnorm, na1 * sizeof(double), cudaMemcpyDeviceToHost,
                                              ctx->stream));
            BEM_TRY(sync_status(ctx));
            std::vector<int> keep;  // positions (in cyc) that run another cycle
            for (int q = 0; q < na1; q++) {
                Col& c = cols[cyc[q]];
                c.cycles++;
                c.rnorm = hnorm[q];
                bool stop = false;
                if (c.rnorm <= c.atol) {
                    stop = true;
                } else if (c.breakdown) {
                    stop = true;
                } else {
                    if (c.presid <= c.ptol)
                        c.ptol_max_factor = std::max(eps, 0.25 * c.ptol_max_factor);
                    else
                        c.ptol_max_factor = std::min(1.0, 1.5 * c.ptol_max_factor);
                    c.ptol = c.presid * std::min(c.ptol_max_factor, c.atol / c.rnorm);
                    if (c.cycles >= maxiter) stop = true;
                }
                if (stop) {
                    c.done = true;
                    c.info = c.rnorm <= c.atol ? 0 : maxiter;
                } else {
                    keep.push_back(q);
                }
            }
            if (!keep.empty() && (int)keep.size() != na1) {
                // compact the residual columns of the continuing columns
                for (size_t q = 0; q < keep.size(); q++) hidx[q] = keep[q];
                BEM_TRY_CUDA(ctx, cudaMemcpyAsync(didx, hidx.data(), keep.size() * sizeof(int), cudaMemcpyHostToDevice,
                                                  ctx->stream));
                gather_kernel<<<nblk((int64_t)n * keep.size()), 256, 0, ctx->stream>>>(T, n, didx, 1.0, P, n,
                                                                                     (int)keep.size());
                BEM_LAUNCHED(ctx);
                std::swap(P, T);
            }
            std::vector<int> ncyc;
            for (int q : keep) ncyc.push_back(cyc[q]);
            cyc.swap(ncyc);
        }
        for (int j = 0; j < nc; j++) {
            const Col& c = cols[j];
            if (iters_out) iters_out[c0 + j] = c.inner;
            if (info_out) info_out[c0 + j] = c.info;
            stats.max_iterations = std::max(stats.max_iterations, c.inner);
            stats.total_iterations += c.inner;
            stats.max_cycles = std::max(stats.max_cycles, c.cycles);
            if (c.bnrm2 > 0) stats.max_rel_residual = std::max(stats.max_rel_residual, c.rnorm / c.bnrm2);
            if (c.info != 0) {
                stats.converged = 0;
                stats.n_unconverged++;
            }
        }
    }
    stats.t_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (st) *st = stats;
    return BEM_OK;
}

static void precond_release(bem_precond* M) {
    if (!M) return;
    cudaSetDevice(M->device);
    for (int i = 0; i < 2; i++) {
        if (M->blk[i]) bem_lu_free(M->blk[i]);
        if (M->blk_z[i]) cudaFree(M->blk_z[i]);
    }
    if (M->dinv) cudaFree(M->dinv);
    delete M;
}

static int precond_create(bem_ctx* ctx, int kind, const void* Zv, int n, int64_t ldz, int precision, bem_lu* lu,
                          bem_precond** out) {
    if (!ctx || !out || n < 1) return fail(ctx, BEM_ERR_INVALID, "bad preconditioner args");
    *out = nullptr;
    const double2* Z = (const double2*)Zv;
    if ((kind == BEM_PRECOND_DIAG || kind == BEM_PRECOND_BLOCK_DIAG) && (!Z || ldz < n))
        return fail(ctx, BEM_ERR_INVALID, "preconditioner needs Z (ldz >= n)");
    if (kind == BEM_PRECOND_LU && (!lu || lu_order(lu) != n))
        return fail(ctx, BEM_ERR_INVALID, "preconditioner factorisation missing or of another order");
    if (kind == BEM_PRECOND_BLOCK_DIAG && (n % 2 != 0))
        return fail(ctx, BEM_ERR_INVALID, "block-diagonal preconditioner needs an even order");
    if (kind < BEM_PRECOND_NONE || kind > BEM_PRECOND_LU)
        return fail(ctx, BEM_ERR_INVALID, "unknown preconditioner kind %d", kind);
    BEM_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    bem_precond* M = new bem_precond();
    M->kind = kind;
    M->n = n;
    M->device = ctx->device;
    int s = BEM_OK;
    if (kind == BEM_PRECOND_LU) {
        M->lu = lu;
    } else if (kind == BEM_PRECOND_DIAG) {
        int* zero = nullptr;
        int hz = 0;
        if (cudaMalloc(&M->dinv, (size_t)n * sizeof(double2)) != cudaSuccess ||
            cudaMalloc(&zero, sizeof(int)) != cudaSuccess) {
            cudaGetLastError();
            s = fail(ctx, BEM_ERR_OOM, "diagonal preconditioner");
        } else {
            cudaMemsetAsync(zero, 0, sizeof(int), ctx->stream);
            inv_diag_kernel<<<(n + 255) / 256, 256, 0, ctx->stream>>>(Z, ldz, n, M->dinv, zero);
            ctx->launches++;
            if (cudaMemcpyAsync(&hz, zero, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
                cudaStreamSynchronize(ctx->stream) != cudaSuccess)
                s = fail(ctx, BEM_ERR_CUDA, "diagonal preconditioner: %s", cudaGetErrorString(cudaGetLastError()));
            else if (hz)
                s = fail(ctx, BEM_ERR_SINGULAR, "diagonal preconditioner: zero diagonal entry");
        }
        if (zero) cudaFree(zero);
    } else if (kind == BEM_PRECOND_BLOCK_DIAG) {
        // LU of Z11 and Z22 (bem_core.py:1147-1158).  The FP64
        // factorisation overwrites its input, so it factors a copy; the FP32
        // one only reads the block, in place in Z (which outlives M as the
        // operator of the solve).
        const int h = n / 2;
        for (int i = 0; i < 2 && s == BEM_OK; i++) {
            double2* blk = const_cast<double2*>(Z) + (int64_t)i * h * ldz + (int64_t)i * h;
            int64_t ldb = ldz;
            if (precision == BEM_PREC_FP64) {
                if (cudaMalloc(&M->blk_z[i], (size_t)h * h * sizeof(double2)) != cudaSuccess) {
                    cudaGetLastError();
                    s = fail(ctx, BEM_ERR_OOM, "block-diagonal preconditioner (%d x %d)", h, h);
                    break;
                }
                copy_block_kernel<<<nblk((int64_t)h * h), 256, 0, ctx->stream>>>(Z, ldz, i * h, h, M->blk_z[i]);
                ctx->launches++;
                blk = M->blk_z[i];
                ldb = h;
            }
            int info = 0;
            s = lu_factor_ex(ctx, blk, h, ldb, precision, false, &M->blk[i], &info);
            if (s == BEM_OK && info != 0)
                s = fail(ctx, BEM_ERR_SINGULAR, "block %d of the preconditioner: U(%d,%d) = 0", i, info, info);
        }
    }
    if (s != BEM_OK) {
        precond_release(M);
        return s;
    }
    *out = M;
    return BEM_OK;
}

}  // namespace bem

using namespace bem;

extern "C" {

int bem_precond_create(bem_ctx* ctx, int kind, const void* Z_dev, int n, int64_t ldz, int precision, bem_lu* lu,
                       bem_precond** out) {
    return precond_create(ctx, kind, Z_dev, n, ldz, precision, lu, out);
}

int bem_precond_free(bem_precond* M) {
    precond_release(M);
    return BEM_OK;
}

int bem_gmres_solve_dev(bem_ctx* ctx, const void* Z_dev, int n, int64_t ldz, bem_precond* M, const void* B_dev,
                        int64_t ldb, void* X_dev, int64_t ldx, int nrhs, int restart, double tol, int maxiter,
                        int* iters, int* info, bem_gmres_stats* stats) {
    if (!ctx || !Z_dev || !M || !B_dev || !X_dev || n < 1 || nrhs < 0 || ldz < n || ldb < n || ldx < n)
        return fail(ctx, BEM_ERR_INVALID, "bad gmres args");
    if (M->n != n) return fail(ctx, BEM_ERR_INVALID, "preconditioner of order %d for a system of order %d", M->n, n);
    if (B_dev == X_dev) return fail(ctx, BEM_ERR_INVALID, "gmres: X must not alias B");
    if (restart < 1 || maxiter < 1 || !(tol > 0))
        return fail(ctx, BEM_ERR_INVALID, "gmres: restart, maxiter >= 1 and tol > 0 required");
    BEM_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    if (nrhs == 0) {
        if (stats) std::memset(stats, 0, sizeof *stats), stats->converged = 1;
        return BEM_OK;
    }
    return gmres_run(ctx, (const double2*)Z_dev, n, ldz, M, (const double2*)B_dev, ldb, (double2*)X_dev, ldx, nrhs,
                     restart, tol, maxiter, iters, info, stats);
}

}  // extern "C"
