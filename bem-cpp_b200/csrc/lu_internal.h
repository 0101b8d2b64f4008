// Shared declarations of the LU / solve / refinement code.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "bem_internal.h"
#include "cgemm_simt.cuh"

namespace bem {

struct PanelWS {
    void* cval;        // 2*G candidate magnitudes (R)
    int* crow;         // 2*G candidate rows
    void* cdata;       // 2*G*w candidate row values
    void* disp;        // 2*w displaced row values
    unsigned* bar;     // grid barrier counter
    int* status;       // sticky status word (BEM_ERR_TIMEOUT on a failed wait)
};

// Optional replacement of the FP64-path GEMM (cgemm) for the big updates
// C -= A * B (A: M x K, K contiguous; B: K x N).  fn: B row-major (the U12
// block of the factor), C row-major.  fn_solve: B and C column-major.
// Options of the three-product tensor-core GEMM C -= op(A) op(B) (complex64).
struct TcOpts {
    bool b_rowmajor = false;  // B is K x N row-major (else given as N x K row-major, "column-major")
    bool c_colmajor = false;  // C column-major
    bool a_trans = false;     // A given as its transpose: K x M row-major
    bool lower = false;       // square row-major C: only the tiles on or below the diagonal
    bool store = false;       // C = -op(A) op(B) (C is not read)
    const float2* bscale = nullptr;  // column-major B: B[k][j] *= bscale[k * bscale_stride]
    int64_t bscale_stride = 0;
    int prof_cls = -1;
};
int tc_gemm_ex(bem_ctx* ctx, int M, int N, int K, const float2* A, int64_t lda, const float2* B, int64_t ldb,
               float2* C, int64_t ldc, const TcOpts& o);

template <typename R> struct TrailingUpdate {
    using C2 = typename C2T<R>::type;
    int (*fn)(bem_ctx*, void*, int M, int N, int K, const C2* A, int64_t lda, const C2* B,
              int64_t ldb, C2* C, int64_t ldc) = nullptr;
    int (*fn_solve)(bem_ctx*, void*, int M, int N, int K, const C2* A, int64_t lda, const C2* B,
                    int64_t ldb, C2* C, int64_t ldc) = nullptr;
    void* state = nullptr;
};

// batch > 1 (FP64 only): `batch` products with the operands offset by sA,
// sB, sC elements per product.
template <typename R>
int cgemm(bem_ctx* ctx, int M, int N, int K, const typename C2T<R>::type* A, int64_t lda,
          const typename C2T<R>::type* B, int64_t ldb, bool b_kmajor,
          typename C2T<R>::type* C, int64_t ldc, bool c_colmajor,
          typename C2T<R>::type alpha, typename C2T<R>::type beta, int prof_cls = -1, int batch = 1,
          int64_t sA = 0, int64_t sB = 0, int64_t sC = 0);

template <typename R>
int getrf(bem_ctx* ctx, typename C2T<R>::type* A, int64_t lda, int n, int* d_ipiv, int* d_info,
          const TrailingUpdate<R>* tc);

template <typename R>
int getrs(bem_ctx* ctx, const typename C2T<R>::type* LU, int64_t lda, int n, const int* d_perm,
          const typename C2T<R>::type* B, int64_t ldb, typename C2T<R>::type* X, int64_t ldx,
          int nrhs, const TrailingUpdate<R>* tc);

void pivots_to_perm(const std::vector<int>& ipiv, std::vector<int>& perm);
// Complex-symmetric S = L D L^T without pivoting (complex64, lower triangle,
// tensor-core updates) and its multi-RHS solve.
int sym_structure(bem_ctx* ctx, const double2* Z, int64_t ldz, int n, bool* sym, bool* sym_half);
constexpr int TRSM_BLOCK = 256;  // rows of the diagonal blocks of the blocked factorisations and solves
// Linv (optional, ceil(n / 256) blocks of 256 x 256): the factorisation
// also stores -L11^-1 of every 256-row diagonal block b at Linv + b 256^2,
// element (r, c) at [c * 256 + r]; the solve then applies the diagonal
// blocks as tensor-core products with these inverses (tmp: 256 x nrhs
// complex64 scratch) instead of block triangular solves.
int sytrf_nopiv(bem_ctx* ctx, float2* A, int64_t lda, int n, int* d_info, float2* Linv = nullptr);
int sytrs_nopiv(bem_ctx* ctx, const float2* A, int64_t lda, int n, const float2* B, int64_t ldb, float2* X,
                int64_t ldx, int nrhs, const float2* Linv = nullptr, float2* tmp = nullptr);

// Factorisation without the int8 digit planes of Z (residual_digits false:
// a factorisation used only as a preconditioner), its order, and one
// application of the factors without refinement (B, X distinct; uses ctx->ws).
int lu_factor_ex(bem_ctx* ctx, void* Z, int n, int64_t ldz, int precision, bool residual_digits, bem_lu** out,
                 int* info);
int lu_order(const bem_lu* lu);
int lu_apply(bem_ctx* ctx, bem_lu* lu, const double2* B, int64_t ldb, double2* X, int64_t ldx, int nrhs);

// Tensor-core updates (gemm_tc.cu: FP16 or TF32 operand parts); nullptr hooks when unavailable.
TrailingUpdate<float> tc_update_fp32(bem_ctx* ctx);

}  // namespace bem
