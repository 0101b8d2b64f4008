// Factorisation objects, FP64 solves and FP32 + FP64-refinement solves,
// and the host-buffer mirrors of solver.h (lu_factorize_cuda, lu_solve_cuda,
// lu_solve_full; solver.cu:7-142).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "bem_internal.h"
#include "lu_internal.h"
#include "ozaki.h"

struct bem_lu {
    bem_ctx* ctx = nullptr;
    int device = 0;
    int n = 0;
    int precision = BEM_PREC_FP64;
    double2* Z = nullptr;   // FP64: the factors (in the caller's buffer); FP32: the original Z
    int64_t ldz = 0;
    float2* A32 = nullptr;  // FP32 factors (owned)
    int* d_ipiv = nullptr;  // owned
    int* d_perm = nullptr;  // owned
    std::vector<int> ipiv;  // 0-based interchange rows
    double znorm = 0.0;     // ||Z||_F
    double t_factor_ms = 0.0;
    bool ldlt = false;      // FP32 factors are L D L^T of Z diag(s) (no pivoting)
    bool dhalf = false;     // s = (I, -I) (else s = 1)
    float2* Linv = nullptr; // L D L^T: -L11^-1 of every 256-row diagonal block (owned; null: block TRSMs)
    size_t linv_bytes = 0;
    float2* stmp = nullptr; // 256 x nrhs scratch of the solves with Linv (owned)
    size_t stmp_bytes = 0;
    bem::OzakiZ oz;         // int8 digit planes of Z for the refinement residual (oz.A null: FP64 GEMM)
};

namespace bem {

// A = complex64(Z), columns >= flip_from negated (flip_from = n: none).
__global__ void z_to_c_kernel(const double2* __restrict__ Z, int64_t ldz, float2* __restrict__ A,
                              int64_t lda, int n, double* __restrict__ fro_part, int flip_from) {
    // one CTA row-block: converts and accumulates |z|^2 into fro_part[blockIdx.x]
    __shared__ double s[256];
    double acc = 0.0;
    int64_t tot = (int64_t)n * n;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < tot;
         i += (int64_t)gridDim.x * blockDim.x) {
        int r = (int)(i / n), c = (int)(i % n);
        double2 z = Z[(int64_t)r * ldz + c];
        acc += z.x * z.x + z.y * z.y;
        if (A) {
            const float sg = c >= flip_from ? -1.f : 1.f;
            A[(int64_t)r * lda + c] = make_float2(sg * (float)z.x, sg * (float)z.y);
        }
    }
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) fro_part[blockIdx.x] = s[0];
}

// per column (column-major n x nrhs): out[c] = max_i |x_ic| (modulus)
template <typename C2>
__global__ void colmax_kernel(const C2* __restrict__ X, int64_t ldx, int n, double* __restrict__ out) {
    __shared__ double s[256];
    const C2* col = X + (int64_t)blockIdx.x * ldx;
    double m = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double a = hypot((double)col[i].x, (double)col[i].y);
        m = fmax(m, a);
    }
    s[threadIdx.x] = m;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) s[threadIdx.x] = fmax(s[threadIdx.x], s[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = s[0];
}

// R32[:, c] = R64[:, c] / scale[c]
__global__ void scale_down_kernel(const double2* __restrict__ R, int64_t ldr, float2* __restrict__ S,
                                  int64_t lds, const double* __restrict__ scale, int n, int nrhs) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)n * nrhs) return;
    int r = (int)(i % n), c = (int)(i / n);
    double sc = scale[c];
    double inv = sc > 0 ? 1.0 / sc : 0.0;
    double2 v = R[(int64_t)c * ldr + r];
    S[(int64_t)c * lds + r] = make_float2((float)(v.x * inv), (float)(v.y * inv));
}

// X[:, c] (+)= scale[c] * D[:, c]
__global__ void scale_up_kernel(const float2* __restrict__ D, int64_t ldd, double2* __restrict__ X,
                                int64_t ldx, const double* __restrict__ scale, int n, int nrhs, int add) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)n * nrhs) return;
    int r = (int)(i % n), c = (int)(i / n);
    double sc = scale[c];
    float2 d = D[(int64_t)c * ldd + r];
    double2* x = &X[(int64_t)c * ldx + r];
    if (add) {
        x->x += sc * (double)d.x;
        x->y += sc * (double)d.y;
    } else {
        *x = make_double2(sc * (double)d.x, sc * (double)d.y);
    }
}

__global__ void copy_cols_kernel(const double2* __restrict__ B, int64_t ldb, double2* __restrict__ X,
                                 int64_t ldx, int n, int nrhs) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)n * nrhs) return;
    int r = (int)(i % n), c = (int)(i / n);
    X[(int64_t)c * ldx + r] = B[(int64_t)c * ldb + r];
}

// Y[:, j] = X[:, idx[j]] (column-major, Y packed with leading dimension n)
__global__ void gather_cols_kernel(const double2* __restrict__ X, int64_t ldx, const int* __restrict__ idx,
                                   double2* __restrict__ Y, int n, int ncols) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)n * ncols) return;
    int r = (int)(i % n), j = (int)(i / n);
    Y[(int64_t)j * n + r] = X[(int64_t)idx[j] * ldx + r];
}

static unsigned nblk(int64_t tot) { return (unsigned)((tot + 255) / 256); }

static int finish_factor(bem_ctx* ctx, bem_lu* lu, int* d_info, int* info) {
    int h[2] = {0, 0};
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(&h[0], d_info, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(&h[1], ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    BEM_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (h[1] != 0) return fail(ctx, h[1], "device-side wait in the panel factorisation gave up");
    lu->ipiv.resize(lu->n);
    BEM_TRY(d2h(ctx, lu->ipiv.data(), lu->d_ipiv, lu->n * sizeof(int)));
    std::vector<int> perm;
    pivots_to_perm(lu->ipiv, perm);
    BEM_TRY(h2d(ctx, lu->d_perm, perm.data(), lu->n * sizeof(int)));
    if (info) *info = h[0];
    return BEM_OK;
}

// X[r][c] = -X[r][c] for r >= r0 (x = diag(I, -I) y)
__global__ void negate_rows_kernel(float2* __restrict__ X, int64_t ldx, int r0, int n, int nrhs) {
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int m = n - r0;
    if (t >= (int64_t)m * nrhs) return;
    const int r = r0 + (int)(t % m), c = (int)(t / m);
    float2 v = X[(int64_t)c * ldx + r];
    X[(int64_t)c * ldx + r] = make_float2(-v.x, -v.y);
}

// D = (FP32 factors)^-1 S for the correction solves.
static int solve32(bem_ctx* ctx, bem_lu* lu, const float2* S, float2* D, int nrhs, const TrailingUpdate<float>* tc) {
    const int n = lu->n;
    if (!lu->ldlt) return getrs<float>(ctx, lu->A32, n, n, lu->d_perm, S, n, D, n, nrhs, tc);
    if (lu->Linv) {
        const size_t need = (size_t)TRSM_BLOCK * nrhs * sizeof(float2);
        if (need > lu->stmp_bytes) {
            if (lu->stmp) {
                BEM_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
                devmem_free(ctx->device, lu->stmp, lu->stmp_bytes, ctx);
            }
            lu->stmp = nullptr;
            lu->stmp_bytes = 0;
            lu->stmp = (float2*)devmem_alloc(ctx->device, need, ctx);
            if (!lu->stmp) return fail(ctx, BEM_ERR_OOM, "solve scratch (%zu bytes)", need);
            lu->stmp_bytes = need;
        }
    }
    BEM_TRY(sytrs_nopiv(ctx, lu->A32, n, n, S, n, D, n, nrhs, lu->Linv, lu->stmp));
    if (lu->dhalf) {
        const int64_t tot = (int64_t)(n - n / 2) * nrhs;
        negate_rows_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, ctx->stream>>>(D, n, n / 2, n, nrhs);
        BEM_LAUNCHED(ctx);
    }
    return BEM_OK;
}

// FP32 LU with partial pivoting of Z into lu->A32 (also the fallback of L D L^T).
static int factor_lu32(bem_ctx* ctx, bem_lu* lu, int* d_info, double* fro, int* info);

// Buffers of the a-posteriori check (all in ctx->ws, sized for nv columns).
struct VerifyWS {
    double2* R;    // n x nv: B - Z X of the checked columns
    double2* X;    // n x nv: the checked columns of X
    float2 *S, *D; // n x nv: scaled residual and its correction
    double *scale, *xmax, *dmax;  // nv each
    int* idx;      // nv column indices
};

// Columns to check: all when nv >= nrhs; else half of them evenly spaced
// over [0, nrhs) and the rest where the last sweep's relative update `upd`
// was largest (the columns furthest from their limit).
static std::vector<int> verify_set(int nrhs, int nv, const std::vector<double>& upd) {
    std::vector<int> idx;
    if (nv >= nrhs) {
        for (int c = 0; c < nrhs; c++) idx.push_back(c);
        return idx;
    }
    std::vector<char> taken(nrhs, 0);
    const int even = (nv + 1) / 2;
    for (int j = 0; j < even; j++) {
        const int c = (int)((int64_t)j * nrhs / even);
        if (!taken[c]) taken[c] = 1, idx.push_back(c);
    }
    std::vector<int> order(nrhs);
    for (int c = 0; c < nrhs; c++) order[c] = c;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return upd[a] > upd[b]; });
    for (int c : order) {
        if ((int)idx.size() >= nv) break;
        if (!taken[c]) taken[c] = 1, idx.push_back(c);
    }
    return idx;
}

// Error of the refined X measured directly on the columns idx: the residual
// r = B - Z x in the FP64 complex GEMM (no digit truncation), then
// e = (FP32 factors)^-1 r.  The factors invert Z to the contraction rho of the
// refinement (~1e-4 here), so |e| is the true error of x to that relative
// accuracy, whatever residual the sweeps used.  *out = max over the checked
// columns of max|e| / max|x|.
static int verify_columns(bem_ctx* ctx, bem_lu* lu, const double2* B, int64_t ldb, const double2* X, int64_t ldx,
                          const std::vector<int>& idx, const VerifyWS& w, const TrailingUpdate<float>* tc,
                          double* out) {
    const int n = lu->n;
    const int nv = (int)idx.size();
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(w.idx, idx.data(), nv * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    const int64_t nn = (int64_t)n * nv;
    gather_cols_kernel<<<nblk(nn), 256, 0, ctx->stream>>>(B, ldb, w.idx, w.R, n, nv);
    BEM_LAUNCHED(ctx);
    gather_cols_kernel<<<nblk(nn), 256, 0, ctx->stream>>>(X, ldx, w.idx, w.X, n, nv);
    BEM_LAUNCHED(ctx);
    BEM_TRY(cgemm<double>(ctx, n, nv, n, lu->Z, lu->ldz, w.X, n, true, w.R, n, true, make_double2(-1, 0),
                          make_double2(1, 0), PROF_VERIFY));
    colmax_kernel<double2><<<nv, 256, 0, ctx->stream>>>(w.R, n, n, w.scale);
    BEM_LAUNCHED(ctx);
    colmax_kernel<double2><<<nv, 256, 0, ctx->stream>>>(w.X, n, n, w.xmax);
    BEM_LAUNCHED(ctx);
    scale_down_kernel<<<nblk(nn), 256, 0, ctx->stream>>>(w.R, n, w.S, n, w.scale, n, nv);
    BEM_LAUNCHED(ctx);
    BEM_TRY(solve32(ctx, lu, w.S, w.D, nv, tc));
    colmax_kernel<float2><<<nv, 256, 0, ctx->stream>>>(w.D, n, n, w.dmax);
    BEM_LAUNCHED(ctx);
    std::vector<double> sc(nv), xm(nv), dm(nv);
    int h_st = 0;
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(sc.data(), w.scale, nv * 8, cudaMemcpyDeviceToHost, ctx->stream));
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(xm.data(), w.xmax, nv * 8, cudaMemcpyDeviceToHost, ctx->stream));
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(dm.data(), w.dmax, nv * 8, cudaMemcpyDeviceToHost, ctx->stream));
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(&h_st, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    BEM_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (h_st != 0) return fail(ctx, h_st, "device-side wait in a tensor-core kernel of the check gave up");
    double e = 0.0;
    for (int j = 0; j < nv; j++) e = std::max(e, sc[j] * dm[j] / (xm[j] > 0 ? xm[j] : 1.0));
    *out = e;
    return BEM_OK;
}

static void lu_release(bem_lu* lu) {
    if (!lu) return;
    cudaSetDevice(lu->device);
    if (lu->A32) bem::devmem_free(lu->device, lu->A32, (size_t)lu->n * lu->n * sizeof(float2), lu->ctx);
    if (lu->Linv) bem::devmem_free(lu->device, lu->Linv, lu->linv_bytes, lu->ctx);
    if (lu->stmp) bem::devmem_free(lu->device, lu->stmp, lu->stmp_bytes, lu->ctx);
    if (lu->d_ipiv) cudaFree(lu->d_ipiv);
    if (lu->d_perm) cudaFree(lu->d_perm);
    bem::ozaki_free(&lu->oz);
    delete lu;
}

static int factor_lu32(bem_ctx* ctx, bem_lu* lu, int* d_info, double* fro, int* info) {
    const int n = lu->n;
    z_to_c_kernel<<<1024, 256, 0, ctx->stream>>>(lu->Z, lu->ldz, lu->A32, n, n, fro, n);
    BEM_LAUNCHED(ctx);
    TrailingUpdate<float> tc = tc_update_fp32(ctx);
    BEM_TRY(getrf<float>(ctx, lu->A32, n, n, lu->d_ipiv, d_info, &tc));
    return finish_factor(ctx, lu, d_info, info);
}

int lu_factor_ex(bem_ctx* ctx, void* Z, int n, int64_t ldz, int precision, bool residual_digits, bem_lu** out,
                 int* info) {
    if (!ctx || !Z || !out || n < 1 || ldz < n) return fail(ctx, BEM_ERR_INVALID, "bad lu_factor args");
    if (precision != BEM_PREC_FP64 && precision != BEM_PREC_FP32_REFINE)
        return fail(ctx, BEM_ERR_INVALID, "unknown precision %d", precision);
    BEM_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    *out = nullptr;
    bem_lu* lu = new bem_lu();
    lu->ctx = ctx;
    lu->device = ctx->device;
    lu->n = n;
    lu->precision = precision;
    lu->Z = (double2*)Z;
    lu->ldz = ldz;
    auto t0 = std::chrono::steady_clock::now();
    int s = BEM_OK;
    int* d_info = nullptr;
    double* fro = nullptr;
    do {
        if (cudaMalloc(&lu->d_ipiv, n * sizeof(int)) != cudaSuccess ||
            cudaMalloc(&lu->d_perm, n * sizeof(int)) != cudaSuccess ||
            cudaMalloc(&d_info, sizeof(int)) != cudaSuccess ||
            cudaMalloc(&fro, 1024 * sizeof(double)) != cudaSuccess) {
            cudaGetLastError();
            s = fail(ctx, BEM_ERR_OOM, "lu workspace");
            break;
        }
        if (precision == BEM_PREC_FP32_REFINE) {
            lu->A32 = (float2*)devmem_alloc(ctx->device, (size_t)n * n * sizeof(float2), ctx);
            if (!lu->A32) {
                s = fail(ctx, BEM_ERR_OOM, "FP32 factor storage (%zu bytes)", (size_t)n * n * sizeof(float2));
                break;
            }
        }
        // symmetric structure: L D L^T without pivoting on Z diag(s)
        if (precision == BEM_PREC_FP32_REFINE && ctx->sym_mode && ctx->use_tc) {
            bool sym = false, sym_half = false;
            s = sym_structure(ctx, lu->Z, ldz, n, &sym, &sym_half);
            if (s != BEM_OK) break;
            lu->ldlt = sym || sym_half;
            lu->dhalf = !sym && sym_half;
        }
        const int flip_from = lu->dhalf ? n / 2 : n;
        z_to_c_kernel<<<1024, 256, 0, ctx->stream>>>(lu->Z, ldz, lu->A32, n, n, fro, flip_from);
        ctx->launches++;
        std::vector<double> hf(1024);
        if (cudaMemcpyAsync(hf.data(), fro, 1024 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
            cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
            s = fail(ctx, BEM_ERR_CUDA, "norm of Z: %s", cudaGetErrorString(cudaGetLastError()));
            break;
        }
        double acc = 0;
        for (double v : hf) acc += v;
        lu->znorm = std::sqrt(acc);
        if (precision == BEM_PREC_FP64) {
            s = getrf<double>(ctx, lu->Z, ldz, n, lu->d_ipiv, d_info, nullptr);
        } else {
            // digit planes of Z for the int8 residual; without room for them the
            // refinement keeps the FP64 tensor-core GEMM
            if (residual_digits && ctx->oz_digits > 0 &&
                ozaki_prepare_z(ctx, &lu->oz, lu->Z, ldz, n, ctx->oz_digits) != BEM_OK)
                ozaki_free(&lu->oz);
            if (lu->ldlt) {
                if (ctx->solve_inv) {
                    // inverses of the diagonal blocks for the solves (without
                    // room for them the solves keep block triangular solves)
                    lu->linv_bytes = (size_t)((n + TRSM_BLOCK - 1) / TRSM_BLOCK) * TRSM_BLOCK * TRSM_BLOCK * sizeof(float2);
                    lu->Linv = (float2*)devmem_alloc(ctx->device, lu->linv_bytes, ctx);
                }
                s = sytrf_nopiv(ctx, lu->A32, n, n, d_info, lu->Linv);
                if (s != BEM_OK) break;
                int h[2] = {0, 0};
                if (cudaMemcpyAsync(&h[0], d_info, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
                    cudaMemcpyAsync(&h[1], ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream) !=
                        cudaSuccess ||
                    cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
                    s = fail(ctx, BEM_ERR_CUDA, "L D L^T: %s", cudaGetErrorString(cudaGetLastError()));
                    break;
                }
                if (h[1] != 0) {
                    s = fail(ctx, h[1], "device-side wait in the L D L^T factorisation gave up");
                    break;
                }
                if (h[0] == 0) {
                    lu->ipiv.resize(n);
                    for (int i = 0; i < n; i++) lu->ipiv[i] = i;
                    if (info) *info = 0;
                    break;
                }
                // a zero pivot without pivoting: partial pivoting instead
                lu->ldlt = lu->dhalf = false;
                if (lu->Linv) devmem_free(ctx->device, lu->Linv, lu->linv_bytes, ctx);
                lu->Linv = nullptr;
            }
            s = factor_lu32(ctx, lu, d_info, fro, info);
            break;
        }
        if (s != BEM_OK) break;
        s = finish_factor(ctx, lu, d_info, info);
    } while (0);
    if (d_info) cudaFree(d_info);
    if (fro) cudaFree(fro);
    if (s != BEM_OK) {
        lu_release(lu);
        return s;
    }
    lu->t_factor_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    *out = lu;
    return BEM_OK;
}

int lu_factor(bem_ctx* ctx, void* Z, int n, int64_t ldz, int precision, bem_lu** out, int* info) {
    return lu_factor_ex(ctx, Z, n, ldz, precision, true, out, info);
}

int lu_order(const bem_lu* lu) { return lu ? lu->n : 0; }

// X = (factors)^-1 B once, without refinement: the FP64 factors' solve, or
// the FP32 factors' solve of B scaled per column by a power of two (the
// first step of the refinement).  B and X distinct.  Uses ctx->ws.
int lu_apply(bem_ctx* ctx, bem_lu* lu, const double2* B, int64_t ldb, double2* X, int64_t ldx, int nrhs) {
    const int n = lu->n;
    if (nrhs <= 0) return BEM_OK;
    if (lu->precision == BEM_PREC_FP64)
        return getrs<double>(ctx, lu->Z, lu->ldz, n, lu->d_perm, B, ldb, X, ldx, nrhs, nullptr);
    const size_t nn = (size_t)n * nrhs;
    size_t off = 0;
    auto take = [&](size_t b) { size_t o = off; off += (b + 255) & ~(size_t)255; return o; };
    size_t o_S = take(nn * sizeof(float2)), o_D = take(nn * sizeof(float2)), o_sc = take(nrhs * sizeof(double));
    BEM_TRY(ctx->ensure_ws(off));
    char* ws = (char*)ctx->ws;
    float2* S = (float2*)(ws + o_S);
    float2* D = (float2*)(ws + o_D);
    double* scale = (double*)(ws + o_sc);
    TrailingUpdate<float> tc = tc_update_fp32(ctx);
    colmax_kernel<double2><<<nrhs, 256, 0, ctx->stream>>>(B, ldb, n, scale);
    BEM_LAUNCHED(ctx);
    scale_down_kernel<<<nblk(nn), 256, 0, ctx->stream>>>(B, ldb, S, n, scale, n, nrhs);
    BEM_LAUNCHED(ctx);
    BEM_TRY(solve32(ctx, lu, S, D, nrhs, &tc));
    scale_up_kernel<<<nblk(nn), 256, 0, ctx->stream>>>(D, n, X, ldx, scale, n, nrhs, 0);
    BEM_LAUNCHED(ctx);
    return BEM_OK;
}

int lu_solve(bem_ctx* ctx, bem_lu* lu, const void* Bv, int64_t ldb, void* Xv, int64_t ldx, int nrhs,
             double tol, int max_iter, bem_solve_stats* st) {
    if (!ctx || !lu || !Bv || !Xv || nrhs < 0 || ldb < lu->n || ldx < lu->n)
        return fail(ctx, BEM_ERR_INVALID, "bad lu_solve args");
    BEM_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    const int n = lu->n;
    const double2* B = (const double2*)Bv;
    double2* X = (double2*)Xv;
    bem_solve_stats stats;
    std::memset(&stats, 0, sizeof stats);
    stats.t_factor_ms = lu->t_factor_ms;
    stats.factorization = lu->precision == BEM_PREC_FP64 ? -1 : lu->ldlt ? (lu->dhalf ? 2 : 1) : 0;
    auto t0 = std::chrono::steady_clock::now();
    if (nrhs == 0) {
        if (st) *st = stats;
        return BEM_OK;
    }
    if (tol <= 0) tol = 1e-11;
    if (max_iter <= 0) max_iter = 10;
    const size_t nn = (size_t)n * nrhs;
    if (lu->precision == BEM_PREC_FP64) {
        // distinct input/output buffers for the row permutation
        const double2* src = B;
        double2* tmp = nullptr;
        if ((const void*)B == (const void*)X) {
            BEM_TRY(ctx->ensure_ws(nn * sizeof(double2)));
            tmp = (double2*)ctx->ws;
            copy_cols_kernel<<<nblk(nn), 256, 0, ctx->stream>>>(B, ldb, tmp, n, n, nrhs);
            BEM_LAUNCHED(ctx);
            src = tmp;
            ldb = n;
        }
        BEM_TRY(getrs<double>(ctx, lu->Z, lu->ldz, n, lu->d_perm, src, ldb, X, ldx, nrhs, nullptr));
        BEM_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        stats.converged = 1;
        stats.t_solve_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        if (st) *st = stats;
        return BEM_OK;
    }
    // FP32 factors + FP64 iterative refinement.
    // workspace: Bc (copy of B when X aliases B), R64, S32, D32, scale, xmax
    size_t off = 0;
    auto take = [&](size_t b) { size_t o = off; off += (b + 255) & ~(size_t)255; return o; };
    bool alias = (const void*)B == (const void*)X;
    size_t o_B = alias ? take(nn * sizeof(double2)) : 0;
    size_t o_R = take(nn * sizeof(double2)), o_S = take(nn * sizeof(float2)), o_D = take(nn * sizeof(float2)),
           o_sc = take(nrhs * sizeof(double)), o_xm = take(nrhs * sizeof(double)),
           o_dm = take(nrhs * sizeof(double));
    // the a-posteriori check reuses R, S, D and the per-column arrays, plus its own copy of the checked columns
    const int nv = ctx->verify_cols < 0 ? nrhs : std::min(ctx->verify_cols, nrhs);
    size_t o_vx = take((size_t)n * std::max(nv, 1) * sizeof(double2)), o_vi = take(std::max(nv, 1) * sizeof(int));
    BEM_TRY(ctx->ensure_ws(off));
    char* ws = (char*)ctx->ws;
    if (alias) {
        double2* Bc = (double2*)(ws + o_B);
        copy_cols_kernel<<<nblk(nn), 256, 0, ctx->stream>>>(B, ldb, Bc, n, n, nrhs);
        BEM_LAUNCHED(ctx);
        B = Bc;
        ldb = n;
    }
    double2* R = (double2*)(ws + o_R);
    float2* S = (float2*)(ws + o_S);
    float2* D = (float2*)(ws + o_D);
    double* scale = (double*)(ws + o_sc);
    double* xmax = (double*)(ws + o_xm);
    double* dmax = (double*)(ws + o_dm);
    TrailingUpdate<float> tc = tc_update_fp32(ctx);
    std::vector<double> h_dm(nrhs), h_xm(nrhs), h_sc(nrhs), col_upd(nrhs, 0.0);
    int h_st = 0;
    BEM_TRY_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream));
    // x0 = (LU32)^-1 B
    colmax_kernel<double2><<<nrhs, 256, 0, ctx->stream>>>(B, ldb, n, scale);
    BEM_LAUNCHED(ctx);
    scale_down_kernel<<<nblk(nn), 256, 0, ctx->stream>>>(B, ldb, S, n, scale, n, nrhs);
    BEM_LAUNCHED(ctx);
    BEM_TRY(solve32(ctx, lu, S, D, nrhs, &tc));
    scale_up_kernel<<<nblk(nn), 256, 0, ctx->stream>>>(D, n, X, ldx, scale, n, nrhs, 0);
    BEM_LAUNCHED(ctx);
    BEM_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    stats.t_solve_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    auto t1 = std::chrono::steady_clock::now();
    double2 m1 = make_double2(-1, 0), p1 = make_double2(1, 0);
    double prev_upd = -1.0;
    // exact: residuals in the FP64 GEMM.  Set from the start without digit
    // planes, and after a check showed the int8 residual's floor (below).
    bool exact = !lu->oz.A;
    bool fresh = false;  // R, D, scale were overwritten by the check: no update form next
    const VerifyWS vws{R, (double2*)(ws + o_vx), S, D, scale, xmax, dmax, (int*)(ws + o_vi)};
    for (int it = 1; it <= max_iter; it++) {
        // R = B - Z X  (FP64 accuracy).  With the int8 digits of Z, sweeps
        // after the first update the previous residual instead,
        // r_k = r_{k-1} - Z d_{k-1}: the correction d is smaller than the
        // iterate by the last relative update, so 7 bits fewer per factor of
        // 128 keep the same absolute accuracy.  One bit of slack: the update
        // form may truncate up to twice as much as the full S-digit product
        // (2^(5-7S) of max|Z| max|x| instead of 2^(4-7S)), still far below
        // the rounding of an FP64 dot product of length n.  The update form
        // carries the first residual's truncation error forward, so the
        // sweeps converge to the solution of Z x = B + (that error): the
        // floor the check after convergence measures.
        int rs = BEM_ERR_OOM;
        if (!exact && it > 1 && prev_upd < 0.5 && !fresh) {
            const double lg = prev_upd > 0 ? -std::log2(prev_upd) + 1.0 : 1e9;
            const int digits = std::min(lu->oz.S, std::max(2, lu->oz.S - (int)std::min(64.0, std::floor(lg / 7.0))));
            // the correction keeps oz_xdigits digits: X, which already holds
            // x + d, becomes x + (d rounded), for which the update is exact
            rs = ozaki_residual_update(ctx, &lu->oz, D, n, scale, R, n, nrhs, digits, ctx->oz_xdigits, X, ldx);
        } else if (!exact) {
            copy_cols_kernel<<<nblk(nn), 256, 0, ctx->stream>>>(B, ldb, R, n, n, nrhs);
            BEM_LAUNCHED(ctx);
            // the first iterate (the FP32 solve's, ~1e-4 relative accuracy) is
            // rounded to oz_xdigits digits (2^-14 of its column's largest entry
            // for 2) and kept so: its residual needs only the digit pairs of
            // those digits, and is exact for it up to Z's digit truncation
            rs = ozaki_residual(ctx, &lu->oz, X, ldx, R, n, nrhs, it == 1 ? ctx->oz_xdigits : 0, it == 1 ? X : nullptr);
        }
        fresh = false;
        if (rs == BEM_ERR_OOM) {
            copy_cols_kernel<<<nblk(nn), 256, 0, ctx->stream>>>(B, ldb, R, n, n, nrhs);
            BEM_LAUNCHED(ctx);
            rs = cgemm<double>(ctx, n, nrhs, n, lu->Z, lu->ldz, X, ldx, true, R, n, true, m1, p1, PROF_RESIDUAL);
            if (lu->oz.A) stats.exact_residual_sweeps++;
        }
        BEM_TRY(rs);
        colmax_kernel<double2><<<nrhs, 256, 0, ctx->stream>>>(R, n, n, scale);
        BEM_LAUNCHED(ctx);
        colmax_kernel<double2><<<nrhs, 256, 0, ctx->stream>>>(X, ldx, n, xmax);
        BEM_LAUNCHED(ctx);
        scale_down_kernel<<<nblk(nn), 256, 0, ctx->stream>>>(R, n, S, n, scale, n, nrhs);
        BEM_LAUNCHED(ctx);
        BEM_TRY(solve32(ctx, lu, S, D, nrhs, &tc));
        colmax_kernel<float2><<<nrhs, 256, 0, ctx->stream>>>(D, n, n, dmax);
        BEM_LAUNCHED(ctx);
        scale_up_kernel<<<nblk(nn), 256, 0, ctx->stream>>>(D, n, X, ldx, scale, n, nrhs, 1);
        BEM_LAUNCHED(ctx);
        BEM_TRY_CUDA(ctx, cudaMemcpyAsync(h_dm.data(), dmax, nrhs * 8, cudaMemcpyDeviceToHost, ctx->stream));
        BEM_TRY_CUDA(ctx, cudaMemcpyAsync(h_xm.data(), xmax, nrhs * 8, cudaMemcpyDeviceToHost, ctx->stream));
        BEM_TRY_CUDA(ctx, cudaMemcpyAsync(h_sc.data(), scale, nrhs * 8, cudaMemcpyDeviceToHost, ctx->stream));
        BEM_TRY_CUDA(ctx, cudaMemcpyAsync(&h_st, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        BEM_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        if (h_st != 0) return fail(ctx, h_st, "device-side wait in a tensor-core kernel of the solve gave up");
        double upd = 0, res = 0;
        for (int c = 0; c < nrhs; c++) {
            double xm = h_xm[c] > 0 ? h_xm[c] : 1.0;
            col_upd[c] = h_sc[c] * h_dm[c] / xm;
            upd = std::max(upd, col_upd[c]);
            res = std::max(res, h_sc[c] / xm);
        }
        stats.iterations = it;
        stats.max_rel_update = upd;
        if (it <= 12) stats.update_hist[it - 1] = upd;
        // max-norm residual relative to ||Z||_F ||x||_max (a bound-style measure)
        stats.max_rel_residual = res / (lu->znorm > 0 ? lu->znorm : 1.0);
        // Error of the new iterate: the sweep contracts the error by rho, so
        // err(x_k) <~ rho / (1 - rho) * |d_k|, with rho estimated from two
        // successive updates (first sweep: assume rho = 0.5, i.e. |d_1|).
        double rho = prev_upd > 0 ? std::min(upd / prev_upd, 0.99) : 0.5;
        double est = upd * rho / (1.0 - rho);
        stats.est_rel_error = est;
        prev_upd = upd;
        if (est <= tol || upd <= 1e-15) {
            // The updates only show how fast the sweeps contract, not the
            // floor left by the residual's own error.  Measure the error
            // directly on nv columns; with a sample (nv < nrhs) the other
            // columns are taken to be within three times the sample's
            // largest (at 2N = 61440 the largest of 2790 columns measured
            // twice the largest of 32 evenly spaced ones).
            if (nv > 0) {
                double ver = 0.0;
                BEM_TRY(verify_columns(ctx, lu, B, ldb, X, ldx, verify_set(nrhs, nv, col_upd), vws, &tc, &ver));
                stats.verified_rel_error = ver;
                stats.verified_columns = nv;
                // checked columns: the factors invert Z only to about the
                // sweep's contraction, so allow 10 % on the measured error
                est = std::max(est, ver * (nv < nrhs ? 3.0 : 1.1));
                stats.est_rel_error = est;
                fresh = true;
            }
            if (est <= tol) {
                stats.converged = 1;
                break;
            }
            // above the tolerance at convergence of the sweeps: the int8
            // residual's floor; recompute the residuals in FP64 from here on
            if (!exact) {
                exact = true;
                prev_upd = -1.0;
                continue;
            }
            if (upd <= 1e-15) break;
        }
    }
    stats.t_refine_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t1).count();
    if (!stats.converged && lu->ldlt) {
        // the factorisation without pivoting was not good enough: partial pivoting, and solve again
        if (alias) {
            copy_cols_kernel<<<nblk(nn), 256, 0, ctx->stream>>>(B, ldb, X, ldx, n, nrhs);
            BEM_LAUNCHED(ctx);
            BEM_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        }
        int* d_info = nullptr;
        double* fro = nullptr;
        if (cudaMalloc(&d_info, sizeof(int)) != cudaSuccess || cudaMalloc(&fro, 1024 * sizeof(double)) != cudaSuccess) {
            cudaGetLastError();
            if (d_info) cudaFree(d_info);
            return fail(ctx, BEM_ERR_OOM, "lu workspace");
        }
        lu->ldlt = lu->dhalf = false;
        if (lu->Linv) devmem_free(ctx->device, lu->Linv, lu->linv_bytes, ctx);
        lu->Linv = nullptr;
        auto tf = std::chrono::steady_clock::now();
        int info = 0;
        int fs = factor_lu32(ctx, lu, d_info, fro, &info);
        cudaFree(d_info);
        cudaFree(fro);
        BEM_TRY(fs);
        if (info > 0) return fail(ctx, BEM_ERR_SINGULAR, "zero pivot at %d", info);
        lu->t_factor_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tf).count();
        return lu_solve(ctx, lu, alias ? (const void*)X : Bv, alias ? ldx : ldb, Xv, ldx, nrhs, tol, max_iter, st);
    }
    if (st) *st = stats;
    if (!stats.converged)
        return fail(ctx, BEM_ERR_NOCONV, "refinement stopped after %d sweeps at relative update %.3e",
                    stats.iterations, stats.max_rel_update);
    return BEM_OK;
}

}  // namespace bem

using namespace bem;

extern "C" {

int bem_lu_factor_dev(bem_ctx* ctx, void* Z_dev, int n, int64_t ldz, int precision, bem_lu** out,
                      int* info) {
    return lu_factor(ctx, Z_dev, n, ldz, precision, out, info);
}

int bem_lu_solve_dev(bem_ctx* ctx, bem_lu* lu, const void* B_dev, int64_t ldb, void* X_dev, int64_t ldx,
                     int nrhs, double tol, int max_iter, bem_solve_stats* stats) {
    return lu_solve(ctx, lu, B_dev, ldb, X_dev, ldx, nrhs, tol, max_iter, stats);
}

int bem_lu_residual_dev(bem_ctx* ctx, bem_lu* lu, const void* B_dev, int64_t ldb, const void* X_dev, int64_t ldx,
                        void* R_dev, int64_t ldr, int nrhs, int method) {
    if (!ctx || !lu || !B_dev || !X_dev || !R_dev || nrhs < 0 || ldb < lu->n || ldx < lu->n || ldr < lu->n)
        return fail(ctx, BEM_ERR_INVALID, "bad lu_residual args");
    if (lu->precision != BEM_PREC_FP32_REFINE)
        return fail(ctx, BEM_ERR_INVALID, "residual needs an FP32_REFINE factorisation (Z kept)");
    if (method == 1 && !lu->oz.A) return fail(ctx, BEM_ERR_INVALID, "factorisation has no int8 digit planes");
    if (method != 0 && method != 1) return fail(ctx, BEM_ERR_INVALID, "unknown residual method %d", method);
    BEM_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    if (nrhs == 0) return BEM_OK;
    const int n = lu->n;
    const double2* X = (const double2*)X_dev;
    double2* R = (double2*)R_dev;
    copy_cols_kernel<<<nblk((int64_t)n * nrhs), 256, 0, ctx->stream>>>((const double2*)B_dev, ldb, R, ldr, n, nrhs);
    BEM_LAUNCHED(ctx);
    BEM_TRY_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream));
    if (method == 1) {
        BEM_TRY(ozaki_residual(ctx, &lu->oz, X, ldx, R, ldr, nrhs));
    } else {
        BEM_TRY(cgemm<double>(ctx, n, nrhs, n, lu->Z, lu->ldz, X, ldx, true, R, ldr, true, make_double2(-1, 0),
                              make_double2(1, 0), PROF_RESIDUAL));
    }
    int h_st = 0;
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(&h_st, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    BEM_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (h_st != 0) return fail(ctx, h_st, "device-side wait in the residual kernel gave up");
    return BEM_OK;
}

int bem_lu_free(bem_lu* lu) {
    lu_release(lu);
    return BEM_OK;
}

// lu_factorize_cuda (solver.cu:7-48): Z host row-major n x n is overwritten
// by the packed factors of P Z = L U; ipiv host, 1-based interchange rows.
int bem_lu_factorize(bem_ctx* ctx, double* Z, int n, int* ipiv, int* info) {
    if (!ctx || !Z || !ipiv || n < 1) return BEM_ERR_INVALID;
    BEM_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    size_t bytes = (size_t)n * n * sizeof(double2);
    void* d = nullptr;
    BEM_TRY_CUDA(ctx, cudaMalloc(&d, bytes));
    bem_lu* lu = nullptr;
    int s = BEM_OK, inf = 0;
    s = h2d(ctx, d, Z, bytes);
    if (s == BEM_OK) s = lu_factor(ctx, d, n, n, BEM_PREC_FP64, &lu, &inf);
    if (s == BEM_OK) s = d2h(ctx, Z, d, bytes);
    if (s == BEM_OK)
        for (int i = 0; i < n; i++) ipiv[i] = lu->ipiv[i] + 1;
    if (lu) lu_release(lu);
    cudaFree(d);
    if (info) *info = inf;
    return s;
}

// lu_solve_cuda (solver.cu:51-84): consumes the pair made by bem_lu_factorize.
int bem_lu_solve(bem_ctx* ctx, const double* Z_lu, const int* ipiv, int n, double* B, int nrhs) {
    if (!ctx || !Z_lu || !ipiv || !B || n < 1 || nrhs < 0) return BEM_ERR_INVALID;
    BEM_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    size_t zb = (size_t)n * n * sizeof(double2), bb = (size_t)n * nrhs * sizeof(double2);
    void *dz = nullptr, *db = nullptr, *dx = nullptr;
    int* dp = nullptr;
    int s = BEM_OK;
    std::vector<int> piv(n), perm;
    for (int i = 0; i < n; i++) {
        piv[i] = ipiv[i] - 1;
        if (piv[i] < 0 || piv[i] >= n) return fail(ctx, BEM_ERR_INVALID, "ipiv[%d] out of range", i);
    }
    pivots_to_perm(piv, perm);
    if (cudaMalloc(&dz, zb) != cudaSuccess || cudaMalloc(&db, bb + 16) != cudaSuccess ||
        cudaMalloc(&dx, bb + 16) != cudaSuccess || cudaMalloc(&dp, n * sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        s = fail(ctx, BEM_ERR_OOM, "lu_solve buffers");
    }
    if (s == BEM_OK) s = h2d(ctx, dz, Z_lu, zb);
    if (s == BEM_OK) s = h2d(ctx, db, B, bb);
    if (s == BEM_OK) s = h2d(ctx, dp, perm.data(), n * sizeof(int));
    if (s == BEM_OK)
        s = getrs<double>(ctx, (const double2*)dz, n, n, dp, (const double2*)db, n, (double2*)dx, n, nrhs, nullptr);
    if (s == BEM_OK) s = d2h(ctx, B, dx, bb);
    cudaFree(dz);
    cudaFree(db);
    cudaFree(dx);
    cudaFree(dp);
    return s;
}

// lu_solve_full (solver.cu:87-142): factor + solve; B (column-major n x nrhs)
// is overwritten with X.  FP64: Z is overwritten with the factors as in the
// reference; FP32_REFINE: Z is left unchanged.
int bem_lu_solve_full(bem_ctx* ctx, double* Z, int n, double* B, int nrhs, int precision,
                      bem_solve_stats* stats) {
    if (!ctx || !Z || !B || n < 1 || nrhs < 0) return BEM_ERR_INVALID;
    BEM_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    size_t zb = (size_t)n * n * sizeof(double2), bb = (size_t)n * nrhs * sizeof(double2);
    void *dz = nullptr, *db = nullptr;
    int s = BEM_OK, info = 0;
    bem_lu* lu = nullptr;
    if (cudaMalloc(&dz, zb) != cudaSuccess || cudaMalloc(&db, bb + 16) != cudaSuccess) {
        cudaGetLastError();
        s = fail(ctx, BEM_ERR_OOM, "lu_solve_full buffers");
    }
    if (s == BEM_OK) s = h2d(ctx, dz, Z, zb);
    if (s == BEM_OK) s = h2d(ctx, db, B, bb);
    if (s == BEM_OK) s = lu_factor(ctx, dz, n, n, precision, &lu, &info);
    if (s == BEM_OK && info > 0) {
        s = fail(ctx, BEM_ERR_SINGULAR, "zero pivot at %d", info);
        if (stats) {
            std::memset(stats, 0, sizeof *stats);
            stats->info = info;
        }
    }
    if (s == BEM_OK) s = lu_solve(ctx, lu, db, n, db, n, nrhs, 0.0, 0, stats);
    if (s == BEM_OK) s = d2h(ctx, B, db, bb);
    if (s == BEM_OK && precision == BEM_PREC_FP64) s = d2h(ctx, Z, dz, zb);
    if (lu) lu_release(lu);
    cudaFree(dz);
    cudaFree(db);
    return s;
}

}  // extern "C"
