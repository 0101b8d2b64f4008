// Complex FP64 GEMM on the FP64 tensor path (mma.sync m8n8k4 f64):
//   C = alpha * A * op(B) + beta * C
// Same operand conventions as cgemm_simt_kernel: A M x K (K contiguous);
// B K x N either K-major (B[j*ldb + k]) or N-major (B[k*ldb + j]); C row- or
// column-major; complex interleaved (double2).
//
// The complex product is taken as two real products over K' = 2K:
//   Re C += A' Bre,  Im C += A' Bim,  A'[i, 2k + p] = (Re, Im) a_ik,
//   Bre[2k + p, j] = (Re b, -Im b)_kj,  Bim[2k + p, j] = (Im b, Re b)_kj,
// so the A fragment of an m8n8k4 step is read straight from the interleaved
// complex row, and one complex B value per thread gives both B fragments.
//
// CTA: 4 warps (2 x 2), 64 x 64 complex outputs, each warp 32 x 32 complex =
// 16 m8n8 tiles for Re and 16 for Im (64 FP64 accumulators per thread).
// K in stages of 16 complex, 2-stage cp.async pipeline (the load of stage
// s + 1 overlaps the products of stage s), 3 CTAs per SM: at the LU update
// shape (M = N = 16384, K = 256, beta = 1) 32.7 TF/s against 30.7 TF/s for
// 3 stages at 2 CTAs per SM; the third resident CTA hides the barrier and
// the epilogue of the others.
//
// zgemm3m_kernel takes the complex product with three real products instead
// of four (Gauss; Higham, "Stability of a method for multiplying complex
// matrices with three real matrix multiplications", SIMAX 13, 1992):
//   T1 = Ar Br,  T2 = Ai Bi,  T3 = (Ar + Ai)(Br + Bi),
//   Re C = T1 - T2,  Im C = T3 - T1 - T2,
// 6MNK real multiply-adds instead of 8MNK.  The error stays normwise at the
// FP64 unit roundoff: |Im error| <= ~K u (|Ar| + |Ai|)(|Br| + |Bi|) instead of
// K u (|Ar||Bi| + |Ai||Br|).  CTA: 8 warps (2 x 4), the same 64 x 64 complex
// tile; each warp 32 x 16 complex with three accumulators (48 FP64 per
// thread); one 128-bit shared load gives a thread both parts of its A (or B)
// fragment element, and the sums Ar + Ai, Br + Bi are formed in registers.
// At M = N = 16384, K = 256, beta = 1: 40.4 (N-major B) / 41.2 (K-major B)
// TF/s counted as 8MNK against 32.2 / 32.5 for zgemm_kernel.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace bem {
namespace dmma {

constexpr int BM = 64, BN = 64, BKC = 16;   // tile, complex K per stage
constexpr int STAGES = 2;
constexpr int AROW = 2 * BKC + 4;           // doubles per A smem row (padded)
constexpr int BROW_K = 2 * BKC + 4;         // doubles per K-major B smem row
constexpr int BROW_N = 2 * BN + 8;          // doubles per N-major B smem row (k row)
constexpr int A_STAGE = BM * AROW;          // doubles
constexpr int B_STAGE_K = BN * BROW_K;
constexpr int B_STAGE_N = BKC * BROW_N;
constexpr int B_STAGE = B_STAGE_K > B_STAGE_N ? B_STAGE_K : B_STAGE_N;
constexpr int SMEM_BYTES = STAGES * (A_STAGE + B_STAGE) * 8;

__device__ __forceinline__ void cp16(void* smem, const void* gmem, bool valid) {
    uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
    int n = valid ? 16 : 0;  // 0: fill with zeros
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(s), "l"(gmem), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

template <bool B_KMAJOR, bool C_COLMAJOR>
__global__ void __launch_bounds__(128, 3)
zgemm_kernel(int M, int N, int K, const double2* __restrict__ A, int64_t lda, const double2* __restrict__ B,
             int64_t ldb, double2* __restrict__ C, int64_t ldc, double2 alpha, double2 beta, int64_t sA = 0,
             int64_t sB = 0, int64_t sC = 0) {
    // a batch of equally shaped products: blockIdx.z selects the matrices
    A += blockIdx.z * sA;
    B += blockIdx.z * sB;
    C += blockIdx.z * sC;
    extern __shared__ __align__(16) double sm[];
    double* As = sm;                          // STAGES x A_STAGE
    double* Bs = sm + STAGES * A_STAGE;       // STAGES x B_STAGE
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;  // warp tile origin (complex)
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int nst = (K + BKC - 1) / BKC;

    // issue the cp.async copies of stage st into buffer buf
    auto load_stage = [&](int st, int buf) {
        const int k0 = st * BKC;
        double* as = As + buf * A_STAGE;
        double* bs = Bs + buf * B_STAGE;
        // A: 64 rows x 16 complex = 1024 copies of 16 B, 8 per thread
#pragma unroll
        for (int l = 0; l < 8; l++) {
            int e = tid + 128 * l;
            int r = e >> 4, kc = e & 15;
            int gi = m0 + r, gk = k0 + kc;
            bool ok = gi < M && gk < K;
            const double2* src = A + (ok ? (int64_t)gi * lda + gk : 0);
            cp16(as + r * AROW + 2 * kc, src, ok);
        }
        if (B_KMAJOR) {
#pragma unroll
            for (int l = 0; l < 8; l++) {
                int e = tid + 128 * l;
                int j = e >> 4, kc = e & 15;
                int gj = n0 + j, gk = k0 + kc;
                bool ok = gj < N && gk < K;
                const double2* src = B + (ok ? (int64_t)gj * ldb + gk : 0);
                cp16(bs + j * BROW_K + 2 * kc, src, ok);
            }
        } else {
#pragma unroll
            for (int l = 0; l < 8; l++) {
                int e = tid + 128 * l;
                int kr = e >> 6, j = e & 63;
                int gj = n0 + j, gk = k0 + kr;
                bool ok = gj < N && gk < K;
                const double2* src = B + (ok ? (int64_t)gk * ldb + gj : 0);
                cp16(bs + kr * BROW_N + 2 * j, src, ok);
            }
        }
    };

    double cre[4][4][2], cim[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) cre[i][j][0] = cre[i][j][1] = cim[i][j][0] = cim[i][j][1] = 0.0;

#pragma unroll
    for (int s = 0; s < STAGES - 1; s++) {
        if (s < nst) load_stage(s, s);
        cp_commit();
    }
    const int fr = lane >> 2, fk = lane & 3;  // fragment row / k' within the m8n8k4 step
    for (int st = 0; st < nst; st++) {
        cp_wait<STAGES - 2>();
        __syncthreads();
        // refill the buffer consumed STAGES-1 stages ago
        {
            int nx = st + STAGES - 1;
            if (nx < nst) load_stage(nx, nx % STAGES);
            cp_commit();
        }
        const int buf = st % STAGES;
        const double* as = As + buf * A_STAGE;
        const double* bs = Bs + buf * B_STAGE;
#pragma unroll
        for (int kk = 0; kk < BKC / 2; kk++) {  // K' steps of 4 (2 complex k)
            double a[4], br[4], bi[4];
#pragma unroll
            for (int i = 0; i < 4; i++) a[i] = as[(wm + 8 * i + fr) * AROW + 4 * kk + fk];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int n = wn + 8 * j + fr, kc = 2 * kk + (fk >> 1);
                double2 b = B_KMAJOR ? *reinterpret_cast<const double2*>(bs + n * BROW_K + 2 * kc)
                                     : *reinterpret_cast<const double2*>(bs + kc * BROW_N + 2 * n);
                br[j] = (fk & 1) ? -b.y : b.x;
                bi[j] = (fk & 1) ? b.x : b.y;
            }
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    dmma(cre[i][j][0], cre[i][j][1], a[i], br[j]);
                    dmma(cim[i][j][0], cim[i][j][1], a[i], bi[j]);
                }
        }
    }
    cp_wait<0>();
    // epilogue: thread holds C(row 8i + lane/4, cols 8j + 2(lane%4) + {0,1})
    const bool has_beta = beta.x != 0.0 || beta.y != 0.0;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int gi = m0 + wm + 8 * i + fr;
        if (gi >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int gj = n0 + wn + 8 * j + 2 * fk + h;
                if (gj >= N) continue;
                const double ar = cre[i][j][h], ai = cim[i][j][h];
                double2 v = make_double2(alpha.x * ar - alpha.y * ai, alpha.x * ai + alpha.y * ar);
                int64_t idx = C_COLMAJOR ? (int64_t)gj * ldc + gi : (int64_t)gi * ldc + gj;
                if (has_beta) {
                    double2 c = C[idx];
                    v.x += beta.x * c.x - beta.y * c.y;
                    v.y += beta.x * c.y + beta.y * c.x;
                }
                C[idx] = v;
            }
    }
}


// ----------------------------------------------------------------- 3M form
constexpr int M3_WM = 2, M3_WN = 4, M3_NJ = 2;  // warps along M / N, 8-column tiles per warp
constexpr int M3_THREADS = 32 * M3_WM * M3_WN;
constexpr int M3_AROW = 2 * BKC + 8;   // doubles: 20 16-byte units, 4 mod 8 (conflict-free 128-bit reads)
constexpr int M3_BROW_K = 2 * BKC + 8;
constexpr int M3_BROW_N = 2 * BN + 4;  // 66 16-byte units, 2 mod 8
constexpr int M3_A_STAGE = BM * M3_AROW;
constexpr int M3_B_STAGE = BN * M3_BROW_K > BKC * M3_BROW_N ? BN * M3_BROW_K : BKC * M3_BROW_N;
constexpr int M3_SMEM_BYTES = STAGES * (M3_A_STAGE + M3_B_STAGE) * 8;
static_assert(32 * M3_WM == BM && 8 * M3_NJ * M3_WN == BN, "3M tile");

template <bool B_KMAJOR, bool C_COLMAJOR>
__global__ void __launch_bounds__(M3_THREADS, 2)
zgemm3m_kernel(int M, int N, int K, const double2* __restrict__ A, int64_t lda, const double2* __restrict__ B,
               int64_t ldb, double2* __restrict__ C, int64_t ldc, double2 alpha, double2 beta, int64_t sA = 0,
               int64_t sB = 0, int64_t sC = 0) {
    constexpr int NJ = M3_NJ;
    A += blockIdx.z * sA;
    B += blockIdx.z * sB;
    C += blockIdx.z * sC;
    extern __shared__ __align__(16) double sm[];
    double* As = sm;                          // STAGES x M3_A_STAGE
    double* Bs = sm + STAGES * M3_A_STAGE;    // STAGES x M3_B_STAGE
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = (warp / M3_WN) * 32, wn = (warp % M3_WN) * 8 * NJ;  // warp tile origin (complex)
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int nst = (K + BKC - 1) / BKC;

    auto load_stage = [&](int st, int buf) {
        const int k0 = st * BKC;
        double* as = As + buf * M3_A_STAGE;
        double* bs = Bs + buf * M3_B_STAGE;
        // A and B: 64 rows x 16 complex each = 1024 copies of 16 B, 4 per thread
#pragma unroll
        for (int l = 0; l < BM * BKC / M3_THREADS; l++) {
            const int e = tid + M3_THREADS * l;
            const int r = e >> 4, kc = e & 15;
            const int gi = m0 + r, gk = k0 + kc;
            const bool ok = gi < M && gk < K;
            cp16(as + r * M3_AROW + 2 * kc, A + (ok ? (int64_t)gi * lda + gk : 0), ok);
        }
#pragma unroll
        for (int l = 0; l < BN * BKC / M3_THREADS; l++) {
            const int e = tid + M3_THREADS * l;
            if (B_KMAJOR) {
                const int j = e >> 4, kc = e & 15;
                const int gj = n0 + j, gk = k0 + kc;
                const bool ok = gj < N && gk < K;
                cp16(bs + j * M3_BROW_K + 2 * kc, B + (ok ? (int64_t)gj * ldb + gk : 0), ok);
            } else {
                const int kr = e >> 6, j = e & 63;
                const int gj = n0 + j, gk = k0 + kr;
                const bool ok = gj < N && gk < K;
                cp16(bs + kr * M3_BROW_N + 2 * j, B + (ok ? (int64_t)gk * ldb + gj : 0), ok);
            }
        }
    };

    double t1[4][NJ][2], t2[4][NJ][2], t3[4][NJ][2];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < NJ; j++)
#pragma unroll
            for (int h = 0; h < 2; h++) t1[i][j][h] = t2[i][j][h] = t3[i][j][h] = 0.0;

#pragma unroll
    for (int s = 0; s < STAGES - 1; s++) {
        if (s < nst) load_stage(s, s);
        cp_commit();
    }
    const int fr = lane >> 2, fk = lane & 3;  // fragment row (A) / column (B), k within the m8n8k4 step
    for (int st = 0; st < nst; st++) {
        cp_wait<STAGES - 2>();
        __syncthreads();
        {
            const int nx = st + STAGES - 1;
            if (nx < nst) load_stage(nx, nx % STAGES);
            cp_commit();
        }
        const int buf = st % STAGES;
        const double* as = As + buf * M3_A_STAGE;
        const double* bs = Bs + buf * M3_B_STAGE;
#pragma unroll
        for (int kk = 0; kk < BKC / 4; kk++) {  // complex K steps of 4
            const int kc = 4 * kk + fk;
            double ar[4], ai[4], asum[4], br[NJ], bi[NJ], bsum[NJ];
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const double2 v = *reinterpret_cast<const double2*>(as + (wm + 8 * i + fr) * M3_AROW + 2 * kc);
                ar[i] = v.x;
                ai[i] = v.y;
                asum[i] = v.x + v.y;
            }
#pragma unroll
            for (int j = 0; j < NJ; j++) {
                const int n = wn + 8 * j + fr;
                const double2 v = B_KMAJOR ? *reinterpret_cast<const double2*>(bs + n * M3_BROW_K + 2 * kc)
                                           : *reinterpret_cast<const double2*>(bs + kc * M3_BROW_N + 2 * n);
                br[j] = v.x;
                bi[j] = v.y;
                bsum[j] = v.x + v.y;
            }
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < NJ; j++) {
                    dmma(t1[i][j][0], t1[i][j][1], ar[i], br[j]);
                    dmma(t2[i][j][0], t2[i][j][1], ai[i], bi[j]);
                    dmma(t3[i][j][0], t3[i][j][1], asum[i], bsum[j]);
                }
        }
    }
    cp_wait<0>();
    // epilogue: thread holds C(row 8i + lane/4, cols 8j + 2(lane%4) + {0,1})
    const bool has_beta = beta.x != 0.0 || beta.y != 0.0;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int gi = m0 + wm + 8 * i + fr;
        if (gi >= M) continue;
#pragma unroll
        for (int j = 0; j < NJ; j++)
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int gj = n0 + wn + 8 * j + 2 * fk + h;
                if (gj >= N) continue;
                const double ar = t1[i][j][h] - t2[i][j][h];
                const double ai = t3[i][j][h] - t1[i][j][h] - t2[i][j][h];
                double2 v = make_double2(alpha.x * ar - alpha.y * ai, alpha.x * ai + alpha.y * ar);
                const int64_t idx = C_COLMAJOR ? (int64_t)gj * ldc + gi : (int64_t)gi * ldc + gj;
                if (has_beta) {
                    const double2 c = C[idx];
                    v.x += beta.x * c.x - beta.y * c.y;
                    v.y += beta.x * c.y + beta.y * c.x;
                }
                C[idx] = v;
            }
    }
}

}  // namespace dmma
}  // namespace bem
