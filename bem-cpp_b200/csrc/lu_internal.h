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

// Optional replacement of the CUDA-core GEMM for the big updates
// C -= A * B (A: M x K, K contiguous; B: K x N).  fn: B row-major (the U12
// block of the factor), C row-major.  fn_solve: B and C column-major.
template <typename R> struct TrailingUpdate {
    using C2 = typename C2T<R>::type;
    int (*fn)(bem_ctx*, void*, int M, int N, int K, const C2* A, int64_t lda, const C2* B,
              int64_t ldb, C2* C, int64_t ldc) = nullptr;
    int (*fn_solve)(bem_ctx*, void*, int M, int N, int K, const C2* A, int64_t lda, const C2* B,
                    int64_t ldb, C2* C, int64_t ldc) = nullptr;
    void* state = nullptr;
};

template <typename R>
int cgemm(bem_ctx* ctx, int M, int N, int K, const typename C2T<R>::type* A, int64_t lda,
          const typename C2T<R>::type* B, int64_t ldb, bool b_kmajor,
          typename C2T<R>::type* C, int64_t ldc, bool c_colmajor,
          typename C2T<R>::type alpha, typename C2T<R>::type beta, int prof_cls = -1);

template <typename R>
int getrf(bem_ctx* ctx, typename C2T<R>::type* A, int64_t lda, int n, int* d_ipiv, int* d_info,
          const TrailingUpdate<R>* tc);

template <typename R>
int getrs(bem_ctx* ctx, const typename C2T<R>::type* LU, int64_t lda, int n, const int* d_perm,
          const typename C2T<R>::type* B, int64_t ldb, typename C2T<R>::type* X, int64_t ldx,
          int nrhs, const TrailingUpdate<R>* tc);

void pivots_to_perm(const std::vector<int>& ipiv, std::vector<int>& perm);

// 3xTF32 tensor-core updates (gemm_tc.cu); nullptr hooks when unavailable.
TrailingUpdate<float> tc_update_fp32(bem_ctx* ctx);

}  // namespace bem
