// Complex GEMM on the CUDA cores, FP64 (DFMA) or FP32 (FFMA):
//   C = alpha * A * op(B) + beta * C
// A is M x K with K contiguous (A[i*lda + k]).  B is K x N given either with K
// contiguous per column (B[j*ldb + k], "K-major") or with N contiguous per row
// (B[k*ldb + j]).  C is row-major (C[i*ldc + j]) or column-major
// (C[j*ldc + i]).  Complex values are interleaved (double2 / float2).
//
// Tiling: 64 x 64 complex outputs per 256-thread CTA, 4 x 4 per thread
// (rows ty + 16 i, columns tx + 16 j, so a warp's shared-memory reads of a
// k-slice touch consecutive 16-byte words), K in steps of BK staged through
// shared memory (double buffered, register prefetch of the next step).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace bem {

template <typename R> struct C2T;
template <> struct C2T<double> { using type = double2; };
template <> struct C2T<float> { using type = float2; };

template <typename C2> __device__ __forceinline__ C2 c2zero() { C2 z; z.x = 0; z.y = 0; return z; }

template <typename R, typename C2>
__device__ __forceinline__ void cfma(C2& acc, const C2 a, const C2 b) {
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(a.y, b.x, acc.y);
}

template <typename R, bool B_KMAJOR, bool C_COLMAJOR>
__global__ void __launch_bounds__(256)
cgemm_simt_kernel(int M, int N, int K, const typename C2T<R>::type* __restrict__ A, int64_t lda,
                  const typename C2T<R>::type* __restrict__ B, int64_t ldb,
                  typename C2T<R>::type* __restrict__ C, int64_t ldc,
                  typename C2T<R>::type alpha, typename C2T<R>::type beta) {
    using C2 = typename C2T<R>::type;
    constexpr int BM = 64, BN = 64;
    constexpr int BK = sizeof(R) == 8 ? 8 : 16;
    constexpr int LA = BM * BK / 256;  // complex loads per thread per operand
    __shared__ C2 As[2][BK][BM + 1];
    __shared__ C2 Bs[2][BK][BN + 1];

    const int tid = threadIdx.x;
    const int tx = tid % 16, ty = tid / 16;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;

    C2 acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = c2zero<C2>();

    C2 ra[LA], rb[LA];
    // loader mapping: element e = tid + 256*l ; K-contiguous tiles read k fastest
    auto load_tiles = [&](int k0) {
#pragma unroll
        for (int l = 0; l < LA; l++) {
            int e = tid + 256 * l;
            int kk = e % BK, r = e / BK;
            int gi = m0 + r, gk = k0 + kk;
            ra[l] = (gi < M && gk < K) ? A[(int64_t)gi * lda + gk] : c2zero<C2>();
            if (B_KMAJOR) {
                int gj = n0 + r;
                rb[l] = (gj < N && gk < K) ? B[(int64_t)gj * ldb + gk] : c2zero<C2>();
            } else {
                int jj = e % BN, kb = e / BN;
                int gj = n0 + jj, gk2 = k0 + kb;
                rb[l] = (gj < N && gk2 < K) ? B[(int64_t)gk2 * ldb + gj] : c2zero<C2>();
            }
        }
    };
    auto store_tiles = [&](int buf) {
#pragma unroll
        for (int l = 0; l < LA; l++) {
            int e = tid + 256 * l;
            int kk = e % BK, r = e / BK;
            As[buf][kk][r] = ra[l];
            if (B_KMAJOR) {
                Bs[buf][kk][r] = rb[l];
            } else {
                int jj = e % BN, kb = e / BN;
                Bs[buf][kb][jj] = rb[l];
            }
        }
    };

    const int nk = (K + BK - 1) / BK;
    load_tiles(0);
    store_tiles(0);
    __syncthreads();
    for (int t = 0; t < nk; t++) {
        const int buf = t & 1;
        if (t + 1 < nk) load_tiles((t + 1) * BK);
#pragma unroll
        for (int kk = 0; kk < BK; kk++) {
            C2 a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; i++) a[i] = As[buf][kk][ty + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; j++) b[j] = Bs[buf][kk][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) cfma<R>(acc[i][j], a[i], b[j]);
        }
        if (t + 1 < nk) store_tiles(buf ^ 1);
        __syncthreads();
    }
    // epilogue: C = alpha*acc + beta*C
    const bool has_beta = (beta.x != 0 || beta.y != 0);
#pragma unroll
    for (int i = 0; i < 4; i++) {
        int gi = m0 + ty + 16 * i;
        if (gi >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            int gj = n0 + tx + 16 * j;
            if (gj >= N) continue;
            int64_t idx = C_COLMAJOR ? (int64_t)gj * ldc + gi : (int64_t)gi * ldc + gj;
            C2 v;
            v.x = alpha.x * acc[i][j].x - alpha.y * acc[i][j].y;
            v.y = alpha.x * acc[i][j].y + alpha.y * acc[i][j].x;
            if (has_beta) {
                C2 c = C[idx];
                v.x += beta.x * c.x - beta.y * c.y;
                v.y += beta.x * c.y + beta.y * c.x;
            }
            C[idx] = v;
        }
    }
}

}  // namespace bem
