// Complex LU with partial pivoting and multi-RHS solves, FP64 and FP32.
//
// Replaces cusolverDnZgetrf / cusolverDnZgetrs (solver.cu:7-142) with a
// blocked right-looking factorisation of the row-major matrix (P Z = L U,
// unit L, LAPACK-style 0-based row pivots kept on the device):
//
//   for each block column of width NB:
//     for each sub-panel of width W inside it:
//       panel_kernel  -- cooperative kernel, whole sub-panel held in shared
//                        memory across all SMs, one grid barrier per column
//                        (pivot search, swap, scale, rank-1 update); panels
//                        that fit the shared memory of one cluster of at
//                        most 8 CTAs run panel_cluster_kernel instead, with
//                        a cluster barrier per column
//       laswp + small TRSM + thin GEMM for the rest of the block column
//     laswp of the block's pivots on the other columns
//     U12 = L11^-1 A12  (blocked TRSM)
//     A22 -= L21 U12    (the trailing update: FP64 on the FP64 tensor path,
//                        mma.sync f64, three real products per complex
//                        one; FP32 on tcgen05 with FP16 (or TF32) parts)
//
// The pivot rule is the one of LAPACK izamax: largest |re| + |im|, first
// index on ties.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "bem_internal.h"
#include "cgemm_simt.cuh"
#include "lu_internal.h"
#include "zgemm_dmma.cuh"

namespace bem {

// ------------------------------------------------------------------- GEMM
template <typename R>
int cgemm(bem_ctx* ctx, int M, int N, int K, const typename C2T<R>::type* A, int64_t lda,
          const typename C2T<R>::type* B, int64_t ldb, bool b_kmajor,
          typename C2T<R>::type* C, int64_t ldc, bool c_colmajor,
          typename C2T<R>::type alpha, typename C2T<R>::type beta, int prof_cls, int batch, int64_t sA,
          int64_t sB, int64_t sC) {
    if (M <= 0 || N <= 0 || batch <= 0) return BEM_OK;
    if (K <= 0) {
        // C = beta*C only; our callers never need it with beta != 1
        return BEM_OK;
    }
    if (batch > 1 && sizeof(R) != 8) return fail(ctx, BEM_ERR_INVALID, "batched GEMM is FP64 only");
    dim3 grid((N + 63) / 64, (M + 63) / 64, batch);
    if (grid.y > 65535) return fail(ctx, BEM_ERR_INVALID, "gemm M too large");
    cudaEvent_t ev = prof_cls >= 0 ? ctx->prof_begin(prof_cls) : nullptr;
    if (sizeof(R) == 8) {
        // FP64: the m8n8k4 f64 tensor path (zgemm_dmma.cuh)
        // the attribute is per device: one bit per (kernel variant, device id)
        // (three real products per complex one unless the context asks for four)
        static std::atomic<unsigned long long> attr[8];
        const double2* Ad = reinterpret_cast<const double2*>(A);
        const double2* Bd = reinterpret_cast<const double2*>(B);
        double2* Cd = reinterpret_cast<double2*>(C);
        double2 al = make_double2(alpha.x, alpha.y), be = make_double2(beta.x, beta.y);
        auto go = [&](auto kern, int slot, int threads, int smem) -> int {
            const unsigned long long bit = 1ull << (ctx->device & 63);
            if (!(attr[slot].load() & bit)) {
                BEM_TRY_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
                attr[slot].fetch_or(bit);
            }
            kern<<<grid, threads, smem, ctx->stream>>>(M, N, K, Ad, lda, Bd, ldb, Cd, ldc, al, be, sA, sB, sC);
            return BEM_OK;
        };
        const int t4 = 128, s4 = dmma::SMEM_BYTES, t3 = dmma::M3_THREADS, s3 = dmma::M3_SMEM_BYTES;
        int s;
        if (ctx->dmma_3m) {
            if (b_kmajor)
                s = c_colmajor ? go(dmma::zgemm3m_kernel<true, true>, 4, t3, s3)
                               : go(dmma::zgemm3m_kernel<true, false>, 5, t3, s3);
            else
                s = c_colmajor ? go(dmma::zgemm3m_kernel<false, true>, 6, t3, s3)
                               : go(dmma::zgemm3m_kernel<false, false>, 7, t3, s3);
        } else if (b_kmajor) {
            s = c_colmajor ? go(dmma::zgemm_kernel<true, true>, 0, t4, s4) : go(dmma::zgemm_kernel<true, false>, 1, t4, s4);
        } else {
            s = c_colmajor ? go(dmma::zgemm_kernel<false, true>, 2, t4, s4)
                           : go(dmma::zgemm_kernel<false, false>, 3, t4, s4);
        }
        BEM_TRY(s);
    } else if (b_kmajor) {
        if (c_colmajor)
            cgemm_simt_kernel<R, true, true><<<grid, 256, 0, ctx->stream>>>(M, N, K, A, lda, B, ldb, C, ldc, alpha, beta);
        else
            cgemm_simt_kernel<R, true, false><<<grid, 256, 0, ctx->stream>>>(M, N, K, A, lda, B, ldb, C, ldc, alpha, beta);
    } else {
        if (c_colmajor)
            cgemm_simt_kernel<R, false, true><<<grid, 256, 0, ctx->stream>>>(M, N, K, A, lda, B, ldb, C, ldc, alpha, beta);
        else
            cgemm_simt_kernel<R, false, false><<<grid, 256, 0, ctx->stream>>>(M, N, K, A, lda, B, ldb, C, ldc, alpha, beta);
    }
    BEM_LAUNCHED(ctx);
    if (ev)
        ctx->prof_end(prof_cls, ev, 8.0 * M * N * K * batch,
                      (double)sizeof(typename C2T<R>::type) * ((double)M * K + (double)K * N + 2.0 * M * N) * batch);
    return BEM_OK;
}

template <typename C2> static C2 mk(double re, double im) {
    C2 c;
    c.x = re;
    c.y = im;
    return c;
}

// ------------------------------------------------------------- grid barrier
// Monotonic arrival counter, reset to 0 before the launch.  Thread 0 of each
// CTA arrives and waits for `target` arrivals, giving up after ~2 s of clock
// cycles (status word := BEM_ERR_TIMEOUT); the kernel then returns.
__device__ __forceinline__ bool grid_barrier(unsigned* bar, unsigned target, int* status,
                                             int* s_flag) {
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        atomicAdd(bar, 1u);
        long long t0 = clock64();
        int ok = 1;
        while (true) {
            unsigned v;
            asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(bar) : "memory");
            if (v >= target) break;
            if (*(volatile int*)status != 0 || clock64() - t0 > 4000000000LL) {
                atomicCAS(status, 0, (int)BEM_ERR_TIMEOUT);
                ok = 0;
                break;
            }
            __nanosleep(20);
        }
        __threadfence();
        *s_flag = ok;
    }
    __syncthreads();
    return *s_flag != 0;
}

template <typename R> __device__ __forceinline__ R cabs1(typename C2T<R>::type v) {
    return fabs(v.x) + fabs(v.y);
}

// ------------------------------------------------------------ panel kernel
// The two per-element operations of a panel column, with explicit fused
// multiply-adds so that every panel kernel rounds them alike:
// l = a inv and x - l u (complex).
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
template <typename C2> __device__ __forceinline__ C2 panel_mul(C2 a, C2 inv) {
    C2 l;
    l.x = fma_rn(a.x, inv.x, -(a.y * inv.y));
    l.y = fma_rn(a.x, inv.y, a.y * inv.x);
    return l;
}
template <typename C2> __device__ __forceinline__ C2 panel_msub(C2 x, C2 l, C2 u) {
    x.x = fma_rn(-l.x, u.x, fma_rn(l.y, u.y, x.x));
    x.y = fma_rn(-l.x, u.y, fma_rn(-l.y, u.x, x.y));
    return x;
}

// Column jj of a panel tile after the interchange: rows below the pivot row
// are scaled by 1/pivot (l = a inv) and the columns right of jj take the
// rank-1 update x -= l u (u: the pivot row).  tpr = w rounded up to a power
// of two threads per row, so a row's threads sit in one warp: they read
// a[i][jj] before the thread of column jj overwrites it with l (__syncwarp),
// with no integer division per element.  Every thread runs the same number
// of passes.
template <typename R>
__device__ __forceinline__ void panel_eliminate(typename C2T<R>::type* tile, int w, int nloc, int lo, int jj,
                                                const typename C2T<R>::type* s_piv, typename C2T<R>::type inv) {
    using C2 = typename C2T<R>::type;
    int tpr = 1;
    while (tpr < w) tpr <<= 1;
    const int rpp = (int)blockDim.x / tpr, cc = (int)threadIdx.x % tpr, i0 = (int)threadIdx.x / tpr;
    const int passes = (nloc + rpp - 1) / rpp;
    C2 u;
    u.x = 0;
    u.y = 0;
    if (cc < w) u = s_piv[cc];
    for (int ps = 0; ps < passes; ps++) {
        const int i = i0 + ps * rpp;
        const bool act = i < nloc && lo + i > jj && cc >= jj && cc < w;
        C2 a;
        a.x = 0;
        a.y = 0;
        if (act) a = tile[i * w + jj];
        const C2 l = panel_mul(a, inv);
        __syncwarp();
        if (act) {
            if (cc == jj)
                tile[i * w + jj] = l;
            else
                tile[i * w + cc] = panel_msub(tile[i * w + cc], l, u);
        }
    }
}

// Factors the sub-panel rows [r0, n), columns [r0, r0+w) of the row-major
// matrix A.  CTA b owns panel rows [b*Rp, min((b+1)*Rp, nrows)) (relative
// to r0) in shared memory; Rp >= w so the w pivot rows live in CTA 0.
// Batched: CTAs [i Gm, (i+1) Gm) factor matrix i (A + i sA, pivots ipiv +
// i sPiv, info + i); every CTA of the grid meets at the one barrier.
template <typename R>
__global__ void __launch_bounds__(256)
panel_kernel(typename C2T<R>::type* __restrict__ A, int64_t lda, int r0, int nrows, int w, int Rp,
             int* __restrict__ ipiv, int* __restrict__ info, PanelWS ws, int Gm, int64_t sA, int sPiv) {
    using C2 = typename C2T<R>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C2* tile = (C2*)smem_raw;                   // Rp * w
    C2* s_piv = tile + (size_t)Rp * w;          // w
    __shared__ R s_val[8];
    __shared__ int s_row[8];
    __shared__ int s_flag;
    __shared__ R s_best;
    __shared__ int s_brow;

    const int G = Gm, mi = blockIdx.x / Gm, b = blockIdx.x % Gm, tid = threadIdx.x;
    const unsigned Gall = gridDim.x;
    A += mi * sA;
    ipiv += mi * sPiv;
    info += mi;
    const int lane = tid & 31, warp = tid >> 5;
    const int lo = b * Rp;
    const int nloc = max(0, min(Rp, nrows - lo));
    R* cval = (R*)ws.cval + (size_t)mi * 2 * Gm;
    int* crow = ws.crow + (size_t)mi * 2 * Gm;
    C2* cdata = (C2*)ws.cdata + (size_t)mi * 2 * Gm * w;
    C2* disp = (C2*)ws.disp + (size_t)mi * 2 * w;

    for (int e = tid; e < nloc * w; e += blockDim.x) {
        int i = e / w, c = e % w;
        tile[e] = A[(int64_t)(r0 + lo + i) * lda + r0 + c];
    }
    __syncthreads();

    for (int jj = 0; jj < w; jj++) {
        const int par = jj & 1;
        // 1. local pivot candidate among rows >= jj
        R bv = (R)-1;
        int br = 0x7fffffff;
        for (int i = tid; i < nloc; i += blockDim.x) {
            int gr = lo + i;
            if (gr < jj) continue;
            R v = cabs1<R>(tile[i * w + jj]);
            if (v > bv || (v == bv && gr < br)) bv = v, br = gr;
        }
        for (int o = 16; o > 0; o >>= 1) {
            R ov = __shfl_down_sync(0xffffffffu, bv, o);
            int orw = __shfl_down_sync(0xffffffffu, br, o);
            if (ov > bv || (ov == bv && orw < br)) bv = ov, br = orw;
        }
        if (lane == 0) s_val[warp] = bv, s_row[warp] = br;
        __syncthreads();
        if (tid == 0) {
            for (int k = 1; k < (int)(blockDim.x >> 5); k++)
                if (s_val[k] > bv || (s_val[k] == bv && s_row[k] < br)) bv = s_val[k], br = s_row[k];
            s_best = bv;
            s_brow = br;
            __stcg(&cval[par * G + b], bv);
            __stcg(&crow[par * G + b], br);
        }
        __syncthreads();
        br = s_brow;
        if (br != 0x7fffffff)
            for (int c = tid; c < w; c += blockDim.x) __stcg(&cdata[((size_t)par * G + b) * w + c], tile[(br - lo) * w + c]);
        if (b == 0)
            for (int c = tid; c < w; c += blockDim.x) __stcg(&disp[par * w + c], tile[jj * w + c]);
        // 2. all candidates published
        if (!grid_barrier(ws.bar, (unsigned)(jj + 1) * Gall, ws.status, &s_flag)) return;
        // 3. global argmax (|re|+|im| max, smallest row on ties); warp 0 also
        // fetches the pivot row
        if (warp == 0) {
            bv = (R)-1;
            br = 0x7fffffff;
            int bo = -1;
            for (int k = lane; k < G; k += 32) {
                R v = __ldcg(&cval[par * G + k]);
                int r = __ldcg(&crow[par * G + k]);
                if (r == 0x7fffffff) continue;
                if (v > bv || (v == bv && r < br)) bv = v, br = r, bo = k;
            }
            for (int o = 16; o > 0; o >>= 1) {
                R ov = __shfl_down_sync(0xffffffffu, bv, o);
                int orw = __shfl_down_sync(0xffffffffu, br, o);
                int oo = __shfl_down_sync(0xffffffffu, bo, o);
                if (ov > bv || (ov == bv && orw < br)) bv = ov, br = orw, bo = oo;
            }
            bv = __shfl_sync(0xffffffffu, bv, 0);
            br = __shfl_sync(0xffffffffu, br, 0);
            bo = __shfl_sync(0xffffffffu, bo, 0);
            const bool zero = !(bv > (R)0);
            if (zero) {
                br = jj;  // no interchange; LAPACK records info and skips the scaling
                bo = -1;
            }
            if (lane < w)
                s_piv[lane] = bo >= 0 ? __ldcg(&cdata[((size_t)par * G + bo) * w + lane]) : __ldcg(&disp[par * w + lane]);
            if (lane == 0) {
                if (zero) atomicCAS(info, 0, r0 + jj + 1);
                s_brow = br;
                s_best = bv;
                if (b == 0) ipiv[r0 + jj] = r0 + br;
            }
        }
        __syncthreads();
        const int piv = s_brow;
        const bool zero = !(s_best > (R)0);
        // 4. interchange rows jj and piv
        if (piv != jj) {
            if (b == 0)
                for (int c = tid; c < w; c += blockDim.x) tile[jj * w + c] = s_piv[c];
            if (piv >= lo && piv < lo + nloc)
                for (int c = tid; c < w; c += blockDim.x) tile[(piv - lo) * w + c] = __ldcg(&disp[par * w + c]);
        }
        __syncthreads();
        // 5. scale column jj below the diagonal, rank-1 update of the rest
        if (!zero) {
            C2 p = s_piv[jj];
            R den = p.x * p.x + p.y * p.y;
            C2 inv;
            inv.x = p.x / den;
            inv.y = -p.y / den;
            panel_eliminate<R>(tile, w, nloc, lo, jj, s_piv, inv);
        }
        __syncthreads();
    }
    for (int e = tid; e < nloc * w; e += blockDim.x) {
        int i = e / w, c = e % w;
        A[(int64_t)(r0 + lo + i) * lda + r0 + c] = tile[e];
    }
}

// ----------------------------------------------------- cluster panel kernel
// The sub-panel of panel_kernel on one thread-block cluster per matrix.  The
// C CTAs of a cluster hold the panel rows in shared memory (CTA b: rows
// [b Rp, (b+1) Rp), Rp >= w, so the w pivot rows live in CTA 0); each
// thread owns whole rows (row pitch WT + 1 complex: no bank conflicts) and is
// the only one to update them.  Per column jj:
//   A. every thread updates its rows for the pivot of column jj (row jj
//      takes the pivot row u, the pivot row takes the former row jj, rows
//      below jj are scaled by 1/u_jj in column jj and take the rank-1 update
//      x -= l u right of it) and keeps the largest |re| + |im| of column
//      jj + 1 among them (smallest row on ties);
//   B. every warp publishes its candidate with that row's values in its
//      CTA's shared memory, CTA 0's owner of row jj + 1 publishes that row;
//   C. cluster barrier;
//   D. warp 0 of every CTA reads the C x 8 candidates through distributed
//      shared memory and reduces them alike: pivot row, its values u, row
//      jj + 1's values, 1/u_jj+1 -- into its own shared memory;
//   E. block barrier.
// One cluster barrier and one block barrier per column, no spin loop.  The
// candidate buffers alternate between two parities: a CTA in column jj + 2
// cannot have passed barrier C of jj + 1 before every CTA has finished step
// D of jj.  Same pivot rule and per-element arithmetic (panel_mul,
// panel_msub) as panel_kernel, so the same pivots and factors.
constexpr int PC_THREADS = 256, PC_WARPS = PC_THREADS / 32;

// The warp's largest bv, the smallest br among the lanes holding it and that
// lane's bk, in every lane.  bv >= 0 (a lane without a candidate holds 0 with
// br = INT_MAX): the bit patterns of non-negative floating-point numbers
// order like unsigned integers, so integer warp reductions find it.
__device__ __forceinline__ void warp_argmax_bits(unsigned hi, unsigned lo, int& br, int& bk, unsigned& mhi,
                                                 unsigned& mlo) {
    mhi = __reduce_max_sync(0xffffffffu, hi);
    mlo = __reduce_max_sync(0xffffffffu, hi == mhi ? lo : 0u);
    const bool top = hi == mhi && lo == mlo;
    const unsigned mrow = __reduce_min_sync(0xffffffffu, top ? (unsigned)br : 0xffffffffu);
    const unsigned win = __ballot_sync(0xffffffffu, top && (unsigned)br == mrow);
    bk = __shfl_sync(0xffffffffu, bk, __ffs(win) - 1);
    br = (int)mrow;
}
__device__ __forceinline__ void warp_argmax(double& bv, int& br, int& bk) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(bv);
    unsigned mhi, mlo;
    warp_argmax_bits((unsigned)(b >> 32), (unsigned)b, br, bk, mhi, mlo);
    bv = __longlong_as_double((long long)(((unsigned long long)mhi << 32) | mlo));
}
__device__ __forceinline__ void warp_argmax(float& bv, int& br, int& bk) {
    unsigned mhi, mlo;
    warp_argmax_bits(__float_as_uint(bv), 0u, br, bk, mhi, mlo);
    bv = __uint_as_float(mhi);
}

template <typename R, int WT>
__global__ void __launch_bounds__(PC_THREADS)
panel_cluster_kernel(typename C2T<R>::type* __restrict__ A, int64_t lda, int r0, int nrows, int w, int Rp,
                     int* __restrict__ ipiv, int* __restrict__ info, int64_t sA, int sPiv) {
    using C2 = typename C2T<R>::type;
    namespace cg = cooperative_groups;
    constexpr int PITCH = WT + 1;
    cg::cluster_group cluster = cg::this_cluster();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C2* tile = (C2*)smem_raw;                          // Rp * PITCH
    C2* pub_data = tile + (size_t)Rp * PITCH;          // [2][PC_WARPS][32]: candidate rows
    C2* disp = pub_data + 2 * PC_WARPS * 32;           // [2][32]: the next pivot row's former values (CTA 0)
    __shared__ R pub_v[2][PC_WARPS];
    __shared__ int pub_row[2][PC_WARPS];
    __shared__ C2 s_u[32], s_dv[32];
    __shared__ C2 s_inv;
    __shared__ int s_piv, s_zero;

    const int C = (int)cluster.num_blocks(), b = (int)cluster.block_rank(), tid = threadIdx.x;
    const int mi = blockIdx.x / C;
    A += mi * sA;
    ipiv += mi * sPiv;
    info += mi;
    const int lane = tid & 31, q = tid >> 5;
    const int lo = b * Rp;
    const int nloc = max(0, min(Rp, nrows - lo));
    const int K = C * PC_WARPS;  // candidates per column
    C2 zero;
    zero.x = 0;
    zero.y = 0;

    for (int e = tid; e < nloc * w; e += blockDim.x) {
        const int i = e / w, c = e % w;
        tile[i * PITCH + c] = A[(int64_t)(r0 + lo + i) * lda + r0 + c];
    }
    __syncthreads();

    // candidate for column 0: every row
    R bv = (R)0;
    int br = 0x7fffffff, bk = 0;
    for (int i = tid; i < nloc; i += PC_THREADS) {
        const R v = cabs1<R>(tile[i * PITCH]);
        if (v > bv || (v == bv && lo + i < br)) bv = v, br = lo + i;
    }

    for (int jn = 0; jn <= w; jn++) {
        // jn >= 1: step A for column jj = jn - 1 (its pivot is in s_*), with
        // the candidate for column jn
        if (jn >= 1) {
            const int jj = jn - 1, piv = s_piv;
            const bool zp = s_zero != 0;
            const C2 inv = s_inv;
            bv = (R)0;
            br = 0x7fffffff;
            for (int i = tid; i < nloc; i += PC_THREADS) {
                const int gr = lo + i;
                C2* row = tile + (size_t)i * PITCH;
                if (gr == jj) {
                    for (int c = 0; c < w; c++) row[c] = s_u[c];
                } else if (gr > jj) {
                    const bool isp = gr == piv && piv != jj;  // takes the former row jj
                    if (isp)
                        for (int c = 0; c < w; c++) row[c] = s_dv[c];
                    if (!zp) {
                        const C2 l = panel_mul(row[jj], inv);
                        row[jj] = l;
                        for (int c = jj + 1; c < w; c++) row[c] = panel_msub(row[c], l, s_u[c]);
                    }
                    if (jn < w) {
                        const R v = cabs1<R>(row[jn]);
                        if (v > bv || (v == bv && gr < br)) bv = v, br = gr;
                    }
                }
            }
        }
        if (jn == w) break;
        const int par = jn & 1;
        // B. publish this warp's candidate for column jn with its row, and row jn
        warp_argmax(bv, br, bk);  // in every lane
        __syncwarp();
        if (lane == 0) {
            pub_v[par][q] = bv;
            pub_row[par][q] = br;
        }
        if (br != 0x7fffffff && lane < w) pub_data[(par * PC_WARPS + q) * 32 + lane] = tile[(br - lo) * PITCH + lane];
        if (b == 0 && (jn % PC_THREADS) / 32 == q && lane < w) disp[par * 32 + lane] = tile[jn * PITCH + lane];
        // C. every candidate of the cluster published (a one-CTA cluster:
        // the block barrier)
        if (C > 1)
            cluster.sync();
        else
            __syncthreads();
        // D. the pivot of column jn, in warp 0 of every CTA
        if (q == 0) {
            R gv = (R)0;
            int grw = 0x7fffffff, gk = -1;
            for (int k = lane; k < K; k += 32) {
                const int rk = k / PC_WARPS, sk = k % PC_WARPS;
                const int r = C > 1 ? *cluster.map_shared_rank(&pub_row[par][sk], rk) : pub_row[par][sk];
                const R v = C > 1 ? *cluster.map_shared_rank(&pub_v[par][sk], rk) : pub_v[par][sk];
                if (r != 0x7fffffff && (v > gv || (v == gv && r < grw))) gv = v, grw = r, gk = k;
            }
            warp_argmax(gv, grw, gk);  // in every lane
            const bool zp = !(gv > (R)0);
            if (zp) {
                grw = jn;  // no interchange; LAPACK records info and skips the scaling
                gk = -1;
            }
            C2 u = zero;
            if (lane < w) {
                const C2* dsrc = C > 1 ? cluster.map_shared_rank(disp, 0) : disp;
                const C2* usrc = C > 1 ? cluster.map_shared_rank(pub_data, gk >= 0 ? gk / PC_WARPS : 0) : pub_data;
                const C2 dv = dsrc[par * 32 + lane];
                u = gk >= 0 ? usrc[(par * PC_WARPS + gk % PC_WARPS) * 32 + lane] : dv;
                s_dv[lane] = dv;
                s_u[lane] = u;
            }
            C2 p;
            p.x = __shfl_sync(0xffffffffu, u.x, jn);
            p.y = __shfl_sync(0xffffffffu, u.y, jn);
            if (lane == 0) {
                C2 inv = zero;
                if (!zp) {
                    const R den = p.x * p.x + p.y * p.y;
                    inv.x = p.x / den;
                    inv.y = -p.y / den;
                }
                s_inv = inv;
                s_piv = grw;
                s_zero = zp ? 1 : 0;
                if (b == 0) {
                    if (zp) atomicCAS(info, 0, r0 + jn + 1);
                    ipiv[r0 + jn] = r0 + grw;
                }
            }
        }
        // E. the pivot known to every thread of this CTA
        __syncthreads();
    }
    __syncthreads();
    for (int e = tid; e < nloc * w; e += blockDim.x) {
        const int i = e / w, c = e % w;
        A[(int64_t)(r0 + lo + i) * lda + r0 + c] = tile[i * PITCH + c];
    }
    // no CTA leaves while another may still read its shared memory
    cluster.sync();
}

constexpr int PANEL_CLUSTER_MAX = 8;                // portable cluster size
constexpr size_t PANEL_CLUSTER_SMEM = 200 * 1024;   // shared memory per CTA

// CTAs per cluster for a sub-panel of nrows x w (elements of `esz` bytes):
// about 384 rows per CTA, every CTA holding at least w rows, at most 8 CTAs
// whose rows fit their shared memory; 0 when the panel does not fit one
// cluster (panel_kernel takes it).
static int panel_cluster_pitch(int w) { return (w <= 8 ? 8 : w <= 16 ? 16 : 32) + 1; }
static size_t panel_cluster_smem(int Rp, int w, size_t esz) {
    return ((size_t)Rp * panel_cluster_pitch(w) + 2 * PC_WARPS * 32 + 2 * 32) * esz;
}
static int panel_cluster_size(int nrows, int w, size_t esz) {
    if (w < 1 || w > 32) return 0;
    int C = std::min(PANEL_CLUSTER_MAX, std::max(1, (nrows + 383) / 384));
    C = std::max(1, std::min(C, nrows / w));
    for (; C <= PANEL_CLUSTER_MAX; C++) {
        const int Rp = (nrows + C - 1) / C;
        if (Rp < w) return 0;
        if (panel_cluster_smem(Rp, w, esz) <= PANEL_CLUSTER_SMEM) return C;
    }
    return 0;
}

// panel_cluster_size, kept only where a cluster of that size and shared
// memory can be resident on this device (cudaOccupancyMaxActiveClusters,
// asked once per shape and remembered); 0: the cooperative panel.
template <typename R>
static int panel_cluster_choice(bem_ctx* ctx, int nrows, int iw) {
    using C2 = typename C2T<R>::type;
    if (!ctx->panel_clusters) return 0;
    const int C = panel_cluster_size(nrows, iw, sizeof(C2));
    if (C < 1) return 0;
    const int Rp = (nrows + C - 1) / C;
    const size_t smem = panel_cluster_smem(Rp, iw, sizeof(C2));
    auto kern = iw <= 8 ? panel_cluster_kernel<R, 8> : iw <= 16 ? panel_cluster_kernel<R, 16> : panel_cluster_kernel<R, 32>;
    static std::mutex mu;
    static std::map<std::tuple<int, const void*, int, size_t>, bool> ok;
    const auto key = std::make_tuple(ctx->device, (const void*)kern, C, (smem + 4095) / 4096);
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = ok.find(key);
        if (it != ok.end()) return it->second ? C : 0;
    }
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PANEL_CLUSTER_SMEM) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)C);
    cfg.blockDim = dim3(PC_THREADS);
    cfg.dynamicSmemBytes = ((smem + 4095) / 4096) * 4096 < PANEL_CLUSTER_SMEM ? ((smem + 4095) / 4096) * 4096 : smem;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)C;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int ncl = 0;
    const bool fits = cudaOccupancyMaxActiveClusters(&ncl, (const void*)kern, &cfg) == cudaSuccess && ncl >= 1;
    if (!fits) cudaGetLastError();
    std::lock_guard<std::mutex> lk(mu);
    ok[key] = fits;
    return fits ? C : 0;
}

// One launch of panel_cluster_kernel: `batch` matrices (A + i sA, pivots
// ipiv + i sPiv, info + i), C CTAs per matrix.
template <typename R>
static int launch_panel_cluster(bem_ctx* ctx, typename C2T<R>::type* A, int64_t lda, int i0, int nrows, int iw,
                                int* d_ipiv, int* d_info, int batch, int64_t sA, int sPiv, int C) {
    using C2 = typename C2T<R>::type;
    static std::atomic<unsigned long long> attr_set{0};
    const unsigned long long bit = 1ull << (ctx->device & 63);
    if (!(attr_set.load() & bit)) {
        BEM_TRY_CUDA(ctx, cudaFuncSetAttribute(panel_cluster_kernel<R, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)PANEL_CLUSTER_SMEM));
        BEM_TRY_CUDA(ctx, cudaFuncSetAttribute(panel_cluster_kernel<R, 16>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PANEL_CLUSTER_SMEM));
        BEM_TRY_CUDA(ctx, cudaFuncSetAttribute(panel_cluster_kernel<R, 32>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PANEL_CLUSTER_SMEM));
        attr_set.fetch_or(bit);
    }
    auto kern = iw <= 8 ? panel_cluster_kernel<R, 8> : iw <= 16 ? panel_cluster_kernel<R, 16> : panel_cluster_kernel<R, 32>;
    const int Rp = (nrows + C - 1) / C;
    const size_t smem = panel_cluster_smem(Rp, iw, sizeof(C2));
    if (smem > PANEL_CLUSTER_SMEM || Rp < iw || iw > 32) return fail(ctx, BEM_ERR_INVALID, "cluster panel bound violated");
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(C * batch));
    cfg.blockDim = dim3(PC_THREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = ctx->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)C;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaEvent_t ev = ctx->prof_begin(PROF_PANEL);
    BEM_TRY_CUDA(ctx, cudaLaunchKernelEx(&cfg, kern, A, lda, i0, nrows, iw, Rp, d_ipiv, d_info, sA, sPiv));
    BEM_LAUNCHED(ctx);
    if (ev)
        ctx->prof_end(PROF_PANEL, ev, 8.0 * (double)nrows * iw * iw / 2 * batch,
                      (double)nrows * iw * 2 * sizeof(C2) * batch);
    return BEM_OK;
}

// ------------------------------------------------------------------ laswp
// Row interchanges k = k0..k1-1 (rows k <-> ipiv[k]) on the columns of up to
// two ranges [c0a, c1a) and [c0b, c1b); one thread per column.
template <typename R>
__global__ void laswp_kernel(typename C2T<R>::type* __restrict__ A, int64_t lda, const int* __restrict__ ipiv,
                             int k0, int k1, int c0a, int c1a, int c0b, int c1b, int64_t sA = 0, int sPiv = 0) {
    using C2 = typename C2T<R>::type;
    A += blockIdx.y * sA;  // batched: blockIdx.y selects the matrix
    ipiv += blockIdx.y * sPiv;
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    int na = c1a - c0a;
    int c;
    if (t < na) c = c0a + t;
    else if (t < na + (c1b - c0b)) c = c0b + (t - na);
    else return;
    for (int k = k0; k < k1; k++) {
        int p = ipiv[k];
        if (p == k) continue;
        C2 x = A[(int64_t)k * lda + c];
        A[(int64_t)k * lda + c] = A[(int64_t)p * lda + c];
        A[(int64_t)p * lda + c] = x;
    }
}

// Row gather for the solve: X[k] = B[perm[k]] for every column (column-major).
template <typename R>
__global__ void permute_rows_kernel(const typename C2T<R>::type* __restrict__ B, int64_t ldb,
                                    typename C2T<R>::type* __restrict__ X, int64_t ldx, const int* __restrict__ perm,
                                    int n, int nrhs, int64_t sB = 0, int64_t sX = 0, int sPerm = 0) {
    B += blockIdx.y * sB;  // batched: blockIdx.y selects the system
    X += blockIdx.y * sX;
    if (perm) perm += blockIdx.y * sPerm;
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)n * nrhs) return;
    int r = (int)(i % n), c = (int)(i / n);
    X[(int64_t)c * ldx + r] = B[(int64_t)c * ldb + (perm ? perm[r] : r)];
}

// ------------------------------------------------------------ small TRSM
// Solves T x = b for one TB x TB diagonal block T = A[r0.., r0..] of the
// row-major factor (UPPER: non-unit upper, backward; else unit lower,
// forward), for every column in [c0, c1) of the right-hand side held either
// row-major in the same matrix (B_ROWMAJOR: element (i, c) at
// B[(r0+i)*ldb + c]) or column-major (B[c*ldb + r0 + i]).  kb <= TB rows.
template <typename R, int TB, bool UPPER, bool B_ROWMAJOR>
__global__ void __launch_bounds__(128)
trsm_small_kernel(const typename C2T<R>::type* __restrict__ T, int64_t ldt, int r0, int kb,
                  typename C2T<R>::type* __restrict__ B, int64_t ldb, int c0, int c1) {
    using C2 = typename C2T<R>::type;
    __shared__ C2 sT[TB][TB + 1];
    for (int e = threadIdx.x; e < kb * kb; e += blockDim.x) {
        int i = e / kb, j = e % kb;
        sT[i][j] = T[(int64_t)(r0 + i) * ldt + r0 + j];
    }
    __syncthreads();
    int c = c0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= c1) return;
    C2 x[TB];
#pragma unroll
    for (int i = 0; i < TB; i++)
        if (i < kb) x[i] = B_ROWMAJOR ? B[(int64_t)(r0 + i) * ldb + c] : B[(int64_t)c * ldb + r0 + i];
    if (!UPPER) {
#pragma unroll
        for (int i = 1; i < TB; i++) {
            if (i >= kb) break;
            C2 s = x[i];
#pragma unroll
            for (int k = 0; k < TB; k++) {
                if (k >= i) break;
                C2 l = sT[i][k];
                s.x -= l.x * x[k].x - l.y * x[k].y;
                s.y -= l.x * x[k].y + l.y * x[k].x;
            }
            x[i] = s;
        }
    } else {
#pragma unroll
        for (int ii = TB - 1; ii >= 0; ii--) {
            if (ii >= kb) continue;
            C2 s = x[ii];
#pragma unroll
            for (int k = 0; k < TB; k++) {
                if (k <= ii || k >= kb) continue;
                C2 u = sT[ii][k];
                s.x -= u.x * x[k].x - u.y * x[k].y;
                s.y -= u.x * x[k].y + u.y * x[k].x;
            }
            C2 d = sT[ii][ii];
            R den = d.x * d.x + d.y * d.y;
            C2 q;
            q.x = (s.x * d.x + s.y * d.y) / den;
            q.y = (s.y * d.x - s.x * d.y) / den;
            x[ii] = q;
        }
    }
#pragma unroll
    for (int i = 0; i < TB; i++)
        if (i < kb) {
            if (B_ROWMAJOR) B[(int64_t)(r0 + i) * ldb + c] = x[i];
            else B[(int64_t)c * ldb + r0 + i] = x[i];
        }
}

template <typename R> struct TBsel { static constexpr int v = 16; };

// ------------------------------------------------------------ block TRSM
// Solves T X = X for a whole diagonal block T = A[r0.., r0..] (kb <= 256 rows;
// UPPER: non-unit upper, backward substitution; else unit lower, forward) in
// one launch, for the columns [c0, c1) of a right-hand side held row-major in
// the factor itself (B_ROWMAJOR, the U12 step) or column-major (the solves).
// One CTA owns RB columns with their kb rows in shared memory (column-major,
// pitch 257) and walks the 16-row diagonal sub-blocks in order: the RB
// threads of the first warps solve the sub-block in registers, then every
// thread updates the one row it owns with the sub-block's 16 solved rows
// (T's row segment in registers, the solved values broadcast from shared
// memory).  This replaces a TRSM + GEMM launch pair per 16 rows.
//
// MODE bits: TRSM_TRANS reads T transposed (T[i][j] = A[r0+j][r0+i], the L^T
// of an L D L^T factor), TRSM_UNIT makes an upper T unit-diagonal, and
// TRSM_DIVDIAG divides the solution of a unit-lower T by T's diagonal (the D
// of L D L^T) when it is stored.
constexpr int TRSM_KB = 256, TRSM_TS = 16, TRSM_PITCH = TRSM_KB + 1;
static_assert(TRSM_KB == TRSM_BLOCK, "diagonal block rows");
constexpr int TRSM_TRANS = 1, TRSM_UNIT = 2, TRSM_DIVDIAG = 4;

template <typename C2> __device__ __forceinline__ C2 cdiv(C2 a, C2 d) {
    const auto den = d.x * d.x + d.y * d.y;
    C2 q;
    q.x = (a.x * d.x + a.y * d.y) / den;
    q.y = (a.y * d.x - a.x * d.y) / den;
    return q;
}

template <typename R, bool UPPER, bool B_ROWMAJOR, int RB, int MODE = 0>
__global__ void __launch_bounds__(TRSM_KB)
trsm_block_kernel(const typename C2T<R>::type* __restrict__ T, int64_t ldt, int r0, int kb,
                  typename C2T<R>::type* __restrict__ B, int64_t ldb, int br0, int c0, int c1, int64_t strideT = 0,
                  int64_t strideB = 0) {
    T += blockIdx.y * strideT;  // batched: blockIdx.y selects the system
    B += blockIdx.y * strideB;
    constexpr bool TRANS = (MODE & TRSM_TRANS) != 0, UNIT = (MODE & TRSM_UNIT) != 0,
                   DIVDIAG = (MODE & TRSM_DIVDIAG) != 0;
    auto tel = [&](int i, int j) {  // element (i, j) of the triangle, block-relative
        return TRANS ? T[(int64_t)(r0 + j) * ldt + r0 + i] : T[(int64_t)(r0 + i) * ldt + r0 + j];
    };
    using C2 = typename C2T<R>::type;
    constexpr int TS = TRSM_TS, XP = TRSM_PITCH;
    extern __shared__ __align__(16) unsigned char trsm_smem[];
    C2* xs = reinterpret_cast<C2*>(trsm_smem);  // xs[c * XP + r]
    __shared__ C2 sT[TS][TS + 1];
    C2 zero;
    zero.x = 0;
    zero.y = 0;
    const int cb = c0 + blockIdx.x * RB;
    const int nc = min(RB, c1 - cb);
    for (int e = threadIdx.x; e < kb * RB; e += blockDim.x) {
        int r, c;
        if (B_ROWMAJOR) {
            r = e / RB;
            c = e % RB;
        } else {
            c = e / kb;
            r = e % kb;
        }
        C2 v = zero;
        if (c < nc) v = B_ROWMAJOR ? B[(int64_t)(br0 + r) * ldb + cb + c] : B[(int64_t)(cb + c) * ldb + br0 + r];
        xs[c * XP + r] = v;
    }
    const int nsb = (kb + TS - 1) / TS;
    for (int step = 0; step < nsb; step++) {
        const int sb = UPPER ? nsb - 1 - step : step;
        const int s0 = sb * TS, ts = min(TS, kb - s0);
        for (int e = threadIdx.x; e < TS * TS; e += blockDim.x) {
            const int i = e / TS, j = e % TS;
            sT[i][j] = (i < ts && j < ts) ? tel(s0 + i, s0 + j) : zero;
        }
        __syncthreads();
        if (threadIdx.x < RB) {
            const int c = threadIdx.x;
            C2 x[TS];
#pragma unroll
            for (int i = 0; i < TS; i++) x[i] = i < ts ? xs[c * XP + s0 + i] : zero;
            if (!UPPER) {
#pragma unroll
                for (int i = 1; i < TS; i++) {
                    C2 acc = x[i];
#pragma unroll
                    for (int k = 0; k < i; k++) {
                        const C2 l = sT[i][k];
                        acc.x -= l.x * x[k].x - l.y * x[k].y;
                        acc.y -= l.x * x[k].y + l.y * x[k].x;
                    }
                    x[i] = acc;
                }
            } else {
#pragma unroll
                for (int ii = TS - 1; ii >= 0; ii--) {
                    if (ii >= ts) continue;
                    C2 acc = x[ii];
#pragma unroll
                    for (int k = ii + 1; k < TS; k++) {
                        const C2 u = sT[ii][k];
                        acc.x -= u.x * x[k].x - u.y * x[k].y;
                        acc.y -= u.x * x[k].y + u.y * x[k].x;
                    }
                    x[ii] = UNIT ? acc : cdiv(acc, sT[ii][ii]);
                }
            }
#pragma unroll
            for (int i = 0; i < TS; i++)
                if (i < ts) xs[c * XP + s0 + i] = x[i];
        }
        __syncthreads();
        const int r = threadIdx.x;
        const bool active = UPPER ? (r < s0) : (r >= s0 + ts && r < kb);
        if (active) {
            C2 t[TS];
#pragma unroll
            for (int m = 0; m < TS; m++) t[m] = m < ts ? tel(r, s0 + m) : zero;
#pragma unroll 4
            for (int c = 0; c < RB; c++) {
                C2 acc = xs[c * XP + r];
#pragma unroll
                for (int m = 0; m < TS; m++) {
                    const C2 y = xs[c * XP + s0 + m];
                    acc.x -= t[m].x * y.x - t[m].y * y.y;
                    acc.y -= t[m].x * y.y + t[m].y * y.x;
                }
                xs[c * XP + r] = acc;
            }
        }
        __syncthreads();
    }
    for (int e = threadIdx.x; e < kb * RB; e += blockDim.x) {
        int r, c;
        if (B_ROWMAJOR) {
            r = e / RB;
            c = e % RB;
        } else {
            c = e / kb;
            r = e % kb;
        }
        if (c < nc) {
            C2 v = xs[c * XP + r];
            if (DIVDIAG) v = cdiv(v, T[(int64_t)(r0 + r) * ldt + r0 + r]);
            if (B_ROWMAJOR) B[(int64_t)(br0 + r) * ldb + cb + c] = v;
            else B[(int64_t)(cb + c) * ldb + br0 + r] = v;
        }
    }
}

// Column-block width of the block TRSM: the factor's U12 rows are wide
// (many columns per CTA amortise the serial sub-block solves), the solves'
// right-hand sides are fewer (more CTAs).  64 KB of shared memory at most.
template <typename R> struct TrsmRB {
    static constexpr int rows_major = sizeof(R) == 4 ? 32 : 16;
    static constexpr int col_major = sizeof(R) == 4 ? 16 : 8;
};

// B's rows of the block start at br0 (at r0, the block's own rows, when br0 < 0).
template <typename R, bool UPPER, bool B_ROWMAJOR, int MODE = 0>
int trsm_block(bem_ctx* ctx, const typename C2T<R>::type* T, int64_t ldt, int r0, int kb,
               typename C2T<R>::type* B, int64_t ldb, int c0, int c1, int br0 = -1, int batch = 1, int64_t sT = 0,
               int64_t sB = 0) {
    if (br0 < 0) br0 = r0;
    using C2 = typename C2T<R>::type;
    constexpr int RB = B_ROWMAJOR ? TrsmRB<R>::rows_major : TrsmRB<R>::col_major;
    if (c1 <= c0 || kb <= 0) return BEM_OK;
    if (kb > TRSM_KB) return fail(ctx, BEM_ERR_INVALID, "block TRSM: %d rows > %d", kb, TRSM_KB);
    const size_t smem = (size_t)RB * TRSM_PITCH * sizeof(C2);
    static_assert(RB * TRSM_PITCH * sizeof(C2) <= 66 * 1024, "block TRSM shared memory");
    // the attribute is per device: one bit per device id, set once
    static std::atomic<unsigned long long> attr_set{0};
    const unsigned long long bit = 1ull << (ctx->device & 63);
    if (!(attr_set.load() & bit)) {
        BEM_TRY_CUDA(ctx, cudaFuncSetAttribute(trsm_block_kernel<R, UPPER, B_ROWMAJOR, RB, MODE>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        attr_set.fetch_or(bit);
    }
    const dim3 grid((c1 - c0 + RB - 1) / RB, batch);
    cudaEvent_t ev = ctx->prof_begin(PROF_TRSM);
    trsm_block_kernel<R, UPPER, B_ROWMAJOR, RB, MODE><<<grid, TRSM_KB, smem, ctx->stream>>>(T, ldt, r0, kb, B, ldb,
                                                                                           br0, c0, c1, sT, sB);
    BEM_LAUNCHED(ctx);
    if (ev)
        ctx->prof_end(PROF_TRSM, ev, 4.0 * kb * (double)kb * (c1 - c0) * batch,
                      (double)sizeof(C2) * ((double)kb * kb / 2 + 2.0 * kb * (c1 - c0)) * batch);
    return BEM_OK;
}

// Unit-lower TRSM on rows [r0, r0+kb) of the row-major matrix itself, for
// columns [c0, c1): the U12 step of the factorisation.
template <typename R>
int trsm_rows_lower_unit(bem_ctx* ctx, typename C2T<R>::type* A, int64_t lda, int r0, int kb,
                         int c0, int c1, int batch = 1, int64_t sA = 0) {
    return trsm_block<R, false, true>(ctx, A, lda, r0, kb, A, lda, c0, c1, -1, batch, sA, sA);
}

// U12 = L11^-1 A12 for the jb x jb unit lower block at (j0, j0), columns
// [c0, n), as a blocked forward substitution: 64-row slabs solved by the
// block triangular solve, each followed by the GEMM update of the slabs
// below (on the FP64 tensor path).  The same arithmetic as the block solve
// of all jb rows, regrouped: three quarters of its flops move to the GEMM.
constexpr int U12_SLAB = 64;
template <typename R>
static int u12_blocked(bem_ctx* ctx, typename C2T<R>::type* A, int64_t lda, int j0, int jb, int c0, int n, int batch,
                       int64_t sA) {
    using C2 = typename C2T<R>::type;
    const int nc = n - c0;
    for (int s0 = 0; s0 < jb; s0 += U12_SLAB) {
        const int sb = std::min(U12_SLAB, jb - s0), below = jb - s0 - sb;
        BEM_TRY(trsm_rows_lower_unit<R>(ctx, A, lda, j0 + s0, sb, c0, n, batch, sA));
        if (below > 0)
            BEM_TRY(cgemm<R>(ctx, below, nc, sb, A + (int64_t)(j0 + s0 + sb) * lda + j0 + s0, lda,
                             A + (int64_t)(j0 + s0) * lda + c0, lda, false, A + (int64_t)(j0 + s0 + sb) * lda + c0, lda,
                             false, mk<C2>(-1, 0), mk<C2>(1, 0), PROF_TRSM, batch, sA, sA, sA));
    }
    return BEM_OK;
}

// ------------------------------------------------------------------ getrf
template <typename R>
int getrf(bem_ctx* ctx, typename C2T<R>::type* A, int64_t lda, int n, int* d_ipiv, int* d_info,
          const TrailingUpdate<R>* tc) {
    using C2 = typename C2T<R>::type;
    const int NB = 256;
    const int W = sizeof(R) == 8 ? 16 : 32;
    // panel workspace
    int occ = 0;
    const int Gmax_sm = ctx->sm_count;
    // rows per CTA for the first (largest) panel decides the shared memory
    // Rows per CTA: ceil(nrows / G) with G = min(SMs, nrows / w); it is at
    // most ceil(n / SMs) while G is capped by the SM count and below 2w
    // once G is nrows / w, so this bounds every panel launch.
    int G0 = std::min(Gmax_sm, std::max(1, n / W));
    int Rp0 = std::max((n + G0 - 1) / G0, 2 * W);
    size_t smem0 = ((size_t)Rp0 * W + W) * sizeof(C2);
    if (smem0 > 220 * 1024)
        return fail(ctx, BEM_ERR_INVALID, "n=%d too large for the panel kernel (%zu B smem)", n, smem0);
    BEM_TRY_CUDA(ctx, cudaFuncSetAttribute(panel_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem0));
    BEM_TRY_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, panel_kernel<R>, 256, smem0));
    if (occ < 1) return fail(ctx, BEM_ERR_INVALID, "panel kernel does not fit on an SM");
    const int Gcap = occ * ctx->sm_count;
    // workspace: cval[2G] (R), crow[2G], cdata[2G*W], disp[2W], bar, status
    size_t ws_bytes = 0;
    auto take = [&](size_t b) { size_t o = ws_bytes; ws_bytes += (b + 255) & ~(size_t)255; return o; };
    size_t o_cval = take(2 * (size_t)Gcap * sizeof(R)), o_crow = take(2 * (size_t)Gcap * 4),
           o_cdata = take(2 * (size_t)Gcap * W * sizeof(C2)), o_disp = take(2 * W * sizeof(C2)),
           o_bar = take(256);
    BEM_TRY(ctx->ensure_ws(ws_bytes));
    char* ws = (char*)ctx->ws;
    PanelWS pw;
    pw.cval = ws + o_cval;
    pw.crow = (int*)(ws + o_crow);
    pw.cdata = ws + o_cdata;
    pw.disp = ws + o_disp;
    pw.bar = (unsigned*)(ws + o_bar);
    pw.status = ctx->d_status;
    BEM_TRY_CUDA(ctx, cudaMemsetAsync(d_info, 0, sizeof(int), ctx->stream));
    BEM_TRY_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream));
    // FP64: U12 = L11^-1 A12 by 64-row slabs with GEMM updates between them
    // (u12_blocked) instead of one block triangular solve of 256 rows
    const bool u12b = sizeof(R) == 8 && ctx->lu_u12_slabs;
    for (int j0 = 0; j0 < n; j0 += NB) {
        const int jb = std::min(NB, n - j0);
        for (int i0 = j0; i0 < j0 + jb; i0 += W) {
            const int iw = std::min(W, j0 + jb - i0);
            const int nrows = n - i0;
            const int Cl = panel_cluster_choice<R>(ctx, nrows, iw);
            if (Cl > 0) {
                BEM_TRY(launch_panel_cluster<R>(ctx, A, lda, i0, nrows, iw, d_ipiv, d_info, 1, 0, 0, Cl));
            } else {
                int G = std::min(Gcap, std::max(1, nrows / iw));
                G = std::min(G, Gmax_sm);
                int Rp = (nrows + G - 1) / G;
                G = (nrows + Rp - 1) / Rp;
                size_t smem = ((size_t)Rp * iw + iw) * sizeof(C2);
                if (smem > smem0) return fail(ctx, BEM_ERR_INVALID, "panel smem bound violated");
                BEM_TRY_CUDA(ctx, cudaMemsetAsync(pw.bar, 0, sizeof(unsigned), ctx->stream));
                int64_t s0 = 0;
                int p0 = 0;
                void* args[] = {&A, (void*)&lda, (void*)&i0, (void*)&nrows, (void*)&iw, (void*)&Rp,
                                &d_ipiv, &d_info, &pw, &G, &s0, &p0};
                cudaEvent_t ev = ctx->prof_begin(PROF_PANEL);
                BEM_TRY_CUDA(ctx, cudaLaunchCooperativeKernel((void*)panel_kernel<R>, dim3(G), dim3(256),
                                                              args, smem, ctx->stream));
                BEM_LAUNCHED(ctx);
                if (ev)
                    ctx->prof_end(PROF_PANEL, ev, 8.0 * (double)nrows * iw * iw / 2,
                                  (double)nrows * iw * 2 * sizeof(C2));
            }
            // interchanges on the rest of this block column
            int ca0 = j0, ca1 = i0, cb0 = i0 + iw, cb1 = j0 + jb;
            int ncol = (ca1 - ca0) + (cb1 - cb0);
            if (ncol > 0) {
                cudaEvent_t ev = ctx->prof_begin(PROF_PIVOT);
                laswp_kernel<R><<<(ncol + 255) / 256, 256, 0, ctx->stream>>>(A, lda, d_ipiv, i0, i0 + iw,
                                                                          ca0, ca1, cb0, cb1);
                BEM_LAUNCHED(ctx);
                if (ev) ctx->prof_end(PROF_PIVOT, ev, 0.0, 4.0 * sizeof(C2) * iw * (double)ncol);
            }
            if (cb1 > cb0) {
                BEM_TRY(trsm_rows_lower_unit<R>(ctx, A, lda, i0, iw, cb0, cb1));
                BEM_TRY(cgemm<R>(ctx, n - i0 - iw, cb1 - cb0, iw, A + (int64_t)(i0 + iw) * lda + i0, lda,
                                 A + (int64_t)i0 * lda + cb0, lda, false,
                                 A + (int64_t)(i0 + iw) * lda + cb0, lda, false, mk<C2>(-1, 0),
                                 mk<C2>(1, 0), PROF_PANEL_UPDATE));
            }
        }
        // interchanges on the columns outside the block column
        int ncol = j0 + (n - j0 - jb);
        if (ncol > 0) {
            cudaEvent_t ev = ctx->prof_begin(PROF_PIVOT);
            laswp_kernel<R><<<(ncol + 255) / 256, 256, 0, ctx->stream>>>(A, lda, d_ipiv, j0, j0 + jb, 0,
                                                                      j0, j0 + jb, n);
            BEM_LAUNCHED(ctx);
            if (ev) ctx->prof_end(PROF_PIVOT, ev, 0.0, 4.0 * sizeof(C2) * jb * (double)ncol);
        }
        const int c0 = j0 + jb;
        if (c0 < n) {
            if (u12b) {
                BEM_TRY(u12_blocked<R>(ctx, A, lda, j0, jb, c0, n, 1, 0));
            } else {
                BEM_TRY(trsm_rows_lower_unit<R>(ctx, A, lda, j0, jb, c0, n));
            }
            const int Mt = n - c0;
            if (tc && tc->fn)
                BEM_TRY(tc->fn(ctx, tc->state, Mt, Mt, jb, A + (int64_t)c0 * lda + j0, lda,
                               A + (int64_t)j0 * lda + c0, lda, A + (int64_t)c0 * lda + c0, lda));
            else
                BEM_TRY(cgemm<R>(ctx, Mt, Mt, jb, A + (int64_t)c0 * lda + j0, lda, A + (int64_t)j0 * lda + c0,
                                 lda, false, A + (int64_t)c0 * lda + c0, lda, false, mk<C2>(-1, 0),
                                 mk<C2>(1, 0), PROF_LU_UPDATE));
        }
    }
    return BEM_OK;
}

// ------------------------------------------------------------------ getrs
// X = (P^T L U)^-1 B, column-major n x nrhs; X may alias B only if perm is
// applied through the workspace (the caller passes distinct buffers).
template <typename R>
int getrs(bem_ctx* ctx, const typename C2T<R>::type* LU, int64_t lda, int n, const int* d_perm,
          const typename C2T<R>::type* B, int64_t ldb, typename C2T<R>::type* X, int64_t ldx,
          int nrhs, const TrailingUpdate<R>* tc) {
    using C2 = typename C2T<R>::type;
    const int NB = 256;
    if (nrhs <= 0) return BEM_OK;
    int64_t tot = (int64_t)n * nrhs;
    permute_rows_kernel<R><<<(unsigned)((tot + 255) / 256), 256, 0, ctx->stream>>>(B, ldb, X, ldx, d_perm,
                                                                                  n, nrhs);
    BEM_LAUNCHED(ctx);
    // forward: L Y = P B
    for (int j0 = 0; j0 < n; j0 += NB) {
        int jb = std::min(NB, n - j0);
        BEM_TRY((trsm_block<R, false, false>(ctx, LU, lda, j0, jb, X, ldx, 0, nrhs)));
        int below = n - j0 - jb;
        if (below > 0) {
            if (tc && tc->fn_solve)
                BEM_TRY(tc->fn_solve(ctx, tc->state, below, nrhs, jb, LU + (int64_t)(j0 + jb) * lda + j0, lda,
                                     X + j0, ldx, X + j0 + jb, ldx));
            else
                BEM_TRY(cgemm<R>(ctx, below, nrhs, jb, LU + (int64_t)(j0 + jb) * lda + j0, lda, X + j0, ldx,
                                 true, X + j0 + jb, ldx, true, mk<C2>(-1, 0), mk<C2>(1, 0), PROF_SOLVE_UPDATE));
        }
    }
    // backward: U X = Y
    int nblk = (n + NB - 1) / NB;
    for (int bi = nblk - 1; bi >= 0; bi--) {
        int j0 = bi * NB, jb = std::min(NB, n - j0);
        BEM_TRY((trsm_block<R, true, false>(ctx, LU, lda, j0, jb, X, ldx, 0, nrhs)));
        if (j0 > 0) {
            if (tc && tc->fn_solve)
                BEM_TRY(tc->fn_solve(ctx, tc->state, j0, nrhs, jb, LU + j0, lda, X + j0, ldx, X, ldx));
            else
                BEM_TRY(cgemm<R>(ctx, j0, nrhs, jb, LU + j0, lda, X + j0, ldx, true, X, ldx, true,
                                 mk<C2>(-1, 0), mk<C2>(1, 0), PROF_SOLVE_UPDATE));
        }
    }
    return BEM_OK;
}

// ------------------------------------------------------------- batched FP64
// The blocked LU of getrf for a batch of equally sized matrices, one launch
// per step for the whole batch.  The panel's CTAs per matrix (Gm) are as many
// as fit co-resident next to the other matrices' (one cooperative grid);
// batches larger than that are factored in chunks.
int getrf_batched(bem_ctx* ctx, double2* A, int64_t lda, int64_t sA, int n, int batch, int* d_ipiv, int* d_info,
                  LuShape shape) {
    using R = double;
    using C2 = double2;
    const int NB = shape.NB, W = shape.W;
    if (n < 1 || batch < 1) return fail(ctx, BEM_ERR_INVALID, "batched LU: n=%d batch=%d", n, batch);
    if (W < 1 || W > 32 || NB < W || NB > TRSM_KB || NB % W != 0)
        return fail(ctx, BEM_ERR_INVALID, "batched LU shape NB=%d W=%d", NB, W);
    const size_t smem_max = 220 * 1024;
    // every sub-panel fits one cluster (the first is the tallest): no
    // cooperative grid, no chunking of the batch
    const bool all_clusters = panel_cluster_choice<R>(ctx, n, W) > 0;
    const int Rp_max = (int)std::min<int64_t>(n, ((int64_t)smem_max / (int64_t)sizeof(C2) - W) / W);
    if (Rp_max < 2 * W) return fail(ctx, BEM_ERR_INVALID, "batched LU: panel does not fit");
    const int Gm_min = (n + Rp_max - 1) / Rp_max;
    // CTAs per matrix for the first panel, and the batch chunk that fits
    int Gm = std::max(Gm_min, std::min(std::max(1, n / W), ctx->sm_count));
    int Rp0 = 0, occ = 0;
    size_t smem0 = 0;
    int chunk = 0;
    BEM_TRY_CUDA(ctx, cudaFuncSetAttribute(panel_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem_max));
    for (;;) {
        Rp0 = std::max((n + Gm - 1) / Gm, 2 * W);
        smem0 = ((size_t)Rp0 * W + W) * sizeof(C2);
        BEM_TRY_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, panel_kernel<R>, 256, smem0));
        if (occ < 1) return fail(ctx, BEM_ERR_INVALID, "batched LU: panel kernel does not fit on an SM");
        chunk = std::min(batch, occ * ctx->sm_count / Gm);
        if (chunk >= batch || Gm == Gm_min) break;
        Gm = std::max(Gm_min, std::min(Gm - 1, occ * ctx->sm_count / batch));
    }
    if (all_clusters) chunk = batch;
    if (chunk < 1) return fail(ctx, BEM_ERR_INVALID, "batched LU: no co-resident panel grid");
    if (chunk < batch) {
        for (int b0 = 0; b0 < batch; b0 += chunk) {
            const int nb = std::min(chunk, batch - b0);
            BEM_TRY(getrf_batched(ctx, A + (int64_t)b0 * sA, lda, sA, n, nb, d_ipiv + (int64_t)b0 * n, d_info + b0,
                                  shape));
        }
        return BEM_OK;
    }
    size_t ws_bytes = 0;
    auto take = [&](size_t b) { size_t o = ws_bytes; ws_bytes += (b + 255) & ~(size_t)255; return o; };
    const size_t per = (size_t)batch * 2 * Gm;
    size_t o_cval = take(per * sizeof(R)), o_crow = take(per * 4), o_cdata = take(per * W * sizeof(C2)),
           o_disp = take((size_t)batch * 2 * W * sizeof(C2)), o_bar = take(256);
    BEM_TRY(ctx->ensure_ws(ws_bytes));
    char* ws = (char*)ctx->ws;
    PanelWS pw;
    pw.cval = ws + o_cval;
    pw.crow = (int*)(ws + o_crow);
    pw.cdata = ws + o_cdata;
    pw.disp = ws + o_disp;
    pw.bar = (unsigned*)(ws + o_bar);
    pw.status = ctx->d_status;
    BEM_TRY_CUDA(ctx, cudaMemsetAsync(d_info, 0, batch * sizeof(int), ctx->stream));
    BEM_TRY_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream));
    const C2 m1 = mk<C2>(-1, 0), p1 = mk<C2>(1, 0);
    // U12 by 64-row slabs, as in getrf (the same arithmetic per matrix)
    const bool u12b = ctx->lu_u12_slabs;
    for (int j0 = 0; j0 < n; j0 += NB) {
        const int jb = std::min(NB, n - j0);
        for (int i0 = j0; i0 < j0 + jb; i0 += W) {
            const int iw = std::min(W, j0 + jb - i0);
            const int nrows = n - i0;
            const int Cl = panel_cluster_choice<R>(ctx, nrows, iw);
            if (Cl > 0) {
                BEM_TRY(launch_panel_cluster<R>(ctx, A, lda, i0, nrows, iw, d_ipiv, d_info, batch, sA, n, Cl));
            } else {
                int G = std::min(Gm, std::max(1, nrows / iw));
                const int Rp = (nrows + G - 1) / G;
                G = (nrows + Rp - 1) / Rp;
                const size_t smem = ((size_t)Rp * iw + iw) * sizeof(C2);
                if (smem > smem0 || Rp < iw) return fail(ctx, BEM_ERR_INVALID, "batched LU: panel bound violated");
                BEM_TRY_CUDA(ctx, cudaMemsetAsync(pw.bar, 0, sizeof(unsigned), ctx->stream));
                int spiv = n;
                void* args[] = {&A, (void*)&lda, (void*)&i0, (void*)&nrows, (void*)&iw, (void*)&Rp,
                                &d_ipiv, &d_info, &pw, &G, &sA, &spiv};
                cudaEvent_t ev = ctx->prof_begin(PROF_PANEL);
                BEM_TRY_CUDA(ctx, cudaLaunchCooperativeKernel((void*)panel_kernel<R>, dim3(G * batch), dim3(256),
                                                              args, smem, ctx->stream));
                BEM_LAUNCHED(ctx);
                if (ev)
                    ctx->prof_end(PROF_PANEL, ev, 8.0 * (double)nrows * iw * iw / 2 * batch,
                                  (double)nrows * iw * 2 * sizeof(C2) * batch);
            }
            const int ca0 = j0, ca1 = i0, cb0 = i0 + iw, cb1 = j0 + jb;
            const int ncol = (ca1 - ca0) + (cb1 - cb0);
            if (ncol > 0) {
                cudaEvent_t ev = ctx->prof_begin(PROF_PIVOT);
                laswp_kernel<R><<<dim3((ncol + 255) / 256, batch), 256, 0, ctx->stream>>>(
                    A, lda, d_ipiv, i0, i0 + iw, ca0, ca1, cb0, cb1, sA, n);
                BEM_LAUNCHED(ctx);
                if (ev) ctx->prof_end(PROF_PIVOT, ev, 0.0, 4.0 * sizeof(C2) * iw * (double)ncol * batch);
            }
            if (cb1 > cb0) {
                BEM_TRY(trsm_rows_lower_unit<R>(ctx, A, lda, i0, iw, cb0, cb1, batch, sA));
                BEM_TRY(cgemm<R>(ctx, n - i0 - iw, cb1 - cb0, iw, A + (int64_t)(i0 + iw) * lda + i0, lda,
                                 A + (int64_t)i0 * lda + cb0, lda, false, A + (int64_t)(i0 + iw) * lda + cb0, lda,
                                 false, m1, p1, PROF_PANEL_UPDATE, batch, sA, sA, sA));
            }
        }
        const int ncol = j0 + (n - j0 - jb);
        if (ncol > 0) {
            cudaEvent_t ev = ctx->prof_begin(PROF_PIVOT);
            laswp_kernel<R><<<dim3((ncol + 255) / 256, batch), 256, 0, ctx->stream>>>(A, lda, d_ipiv, j0, j0 + jb, 0,
                                                                                      j0, j0 + jb, n, sA, n);
            BEM_LAUNCHED(ctx);
            if (ev) ctx->prof_end(PROF_PIVOT, ev, 0.0, 4.0 * sizeof(C2) * jb * (double)ncol * batch);
        }
        const int c0 = j0 + jb;
        if (c0 < n) {
            if (u12b)
                BEM_TRY(u12_blocked<R>(ctx, A, lda, j0, jb, c0, n, batch, sA));
            else
                BEM_TRY(trsm_rows_lower_unit<R>(ctx, A, lda, j0, jb, c0, n, batch, sA));
            const int Mt = n - c0;
            BEM_TRY(cgemm<R>(ctx, Mt, Mt, jb, A + (int64_t)c0 * lda + j0, lda, A + (int64_t)j0 * lda + c0, lda, false,
                             A + (int64_t)c0 * lda + c0, lda, false, m1, p1, PROF_LU_UPDATE, batch, sA, sA, sA));
        }
    }
    return BEM_OK;
}

int getrs_batched(bem_ctx* ctx, const double2* LU, int64_t lda, int64_t sA, int n, int batch, const int* d_perm,
                  const double2* B, int64_t ldb, int64_t sB, double2* X, int64_t ldx, int64_t sX, int nrhs, int NB) {
    using R = double;
    using C2 = double2;
    if (nrhs <= 0 || batch <= 0) return BEM_OK;
    if (NB < 1 || NB > TRSM_KB) return fail(ctx, BEM_ERR_INVALID, "batched solve block %d", NB);
    const int64_t tot = (int64_t)n * nrhs;
    permute_rows_kernel<R><<<dim3((unsigned)((tot + 255) / 256), batch), 256, 0, ctx->stream>>>(
        B, ldb, X, ldx, d_perm, n, nrhs, sB, sX, n);
    BEM_LAUNCHED(ctx);
    const C2 m1 = mk<C2>(-1, 0), p1 = mk<C2>(1, 0);
    for (int j0 = 0; j0 < n; j0 += NB) {
        const int jb = std::min(NB, n - j0);
        BEM_TRY((trsm_block<R, false, false>(ctx, LU, lda, j0, jb, X, ldx, 0, nrhs, -1, batch, sA, sX)));
        const int below = n - j0 - jb;
        if (below > 0)
            BEM_TRY(cgemm<R>(ctx, below, nrhs, jb, LU + (int64_t)(j0 + jb) * lda + j0, lda, X + j0, ldx, true,
                             X + j0 + jb, ldx, true, m1, p1, PROF_SOLVE_UPDATE, batch, sA, sX, sX));
    }
    const int nblk = (n + NB - 1) / NB;
    for (int bi = nblk - 1; bi >= 0; bi--) {
        const int j0 = bi * NB, jb = std::min(NB, n - j0);
        BEM_TRY((trsm_block<R, true, false>(ctx, LU, lda, j0, jb, X, ldx, 0, nrhs, -1, batch, sA, sX)));
        if (j0 > 0)
            BEM_TRY(cgemm<R>(ctx, j0, nrhs, jb, LU + j0, lda, X + j0, ldx, true, X, ldx, true, m1, p1,
                             PROF_SOLVE_UPDATE, batch, sA, sX, sX));
    }
    return BEM_OK;
}

// Deterministic fill of a batch of test matrices for the autotuner: entries
// in [-1, 1) from an integer hash, plus n on the diagonal.
static __global__ void tune_fill_kernel(double2* A, int n, int64_t total) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    uint64_t h = (uint64_t)i * 0x9E3779B97F4A7C15ull;
    h ^= h >> 31;
    h *= 0xBF58476D1CE4E5B9ull;
    h ^= h >> 29;
    const double re = (double)(h & 0xFFFFFF) / 8388608.0 - 1.0, im = (double)((h >> 24) & 0xFFFFFF) / 8388608.0 - 1.0;
    const int64_t e = i % ((int64_t)n * n);
    const bool diag = e / n == e % n;
    A[i] = make_double2(re + (diag ? n : 0.0), im);
}

// Shape of the batched FP64 LU for (n, batch): every candidate block / panel
// width is timed once (after one warm-up) on min(batch, 8) test matrices of
// order n, and the fastest kept for the context's later batches of that
// shape.
int tune_lu_shape(bem_ctx* ctx, int n, int batch, LuShape* out) {
    static std::map<std::pair<int, int>, LuShape> cache;  // per process: (n, batch) -> shape
    const int tb = std::min(batch, 8);
    const auto key = std::make_pair(n, tb);
    auto it = cache.find(key);
    if (it != cache.end()) {
        *out = it->second;
        return BEM_OK;
    }
    const LuShape cands[] = {{256, 16}, {128, 16}, {256, 32}, {128, 32}, {256, 8}, {64, 16}};
    const size_t nn = (size_t)n * n;
    void* A = devmem_alloc(ctx->device, nn * tb * sizeof(double2), ctx);
    void* ip = devmem_alloc(ctx->device, (size_t)n * tb * sizeof(int) + (size_t)tb * sizeof(int), ctx);
    if (!A || !ip) {
        if (A) devmem_free(ctx->device, A, nn * tb * sizeof(double2), ctx);
        if (ip) devmem_free(ctx->device, ip, (size_t)n * tb * sizeof(int) + (size_t)tb * sizeof(int), ctx);
        *out = LuShape{};
        return BEM_OK;  // no room to tune: the default shape
    }
    int* d_ipiv = (int*)ip;
    int* d_info = d_ipiv + (size_t)n * tb;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    LuShape pick{};
    int s = BEM_OK;
    for (const LuShape& c : cands) {
        if (c.NB > n && c.NB != 256) continue;
        float ms = 0.f;
        for (int rep = 0; rep < 2 && s == BEM_OK; rep++) {
            const int64_t tot = (int64_t)nn * tb;
            tune_fill_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, ctx->stream>>>((double2*)A, n, tot);
            ctx->launches++;
            cudaEventRecord(e0, ctx->stream);
            s = getrf_batched(ctx, (double2*)A, n, (int64_t)nn, n, tb, d_ipiv, d_info, c);
            cudaEventRecord(e1, ctx->stream);
            if (cudaEventSynchronize(e1) != cudaSuccess) s = fail(ctx, BEM_ERR_CUDA, "LU autotuner");
            cudaEventElapsedTime(&ms, e0, e1);
        }
        if (s != BEM_OK) break;
        if (ms < best) best = ms, pick = c;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    devmem_free(ctx->device, A, nn * tb * sizeof(double2), ctx);
    devmem_free(ctx->device, ip, (size_t)n * tb * sizeof(int) + (size_t)tb * sizeof(int), ctx);
    if (s != BEM_OK) return s;
    cache[key] = pick;
    *out = pick;
    return BEM_OK;
}

template int getrf<double>(bem_ctx*, double2*, int64_t, int, int*, int*, const TrailingUpdate<double>*);
template int getrf<float>(bem_ctx*, float2*, int64_t, int, int*, int*, const TrailingUpdate<float>*);
template int getrs<double>(bem_ctx*, const double2*, int64_t, int, const int*, const double2*, int64_t,
                           double2*, int64_t, int, const TrailingUpdate<double>*);
template int getrs<float>(bem_ctx*, const float2*, int64_t, int, const int*, const float2*, int64_t,
                          float2*, int64_t, int, const TrailingUpdate<float>*);
template int cgemm<double>(bem_ctx*, int, int, int, const double2*, int64_t, const double2*, int64_t, bool,
                           double2*, int64_t, bool, double2, double2, int, int, int64_t, int64_t, int64_t);
template int cgemm<float>(bem_ctx*, int, int, int, const float2*, int64_t, const float2*, int64_t, bool,
                          float2*, int64_t, bool, float2, float2, int, int, int64_t, int64_t, int64_t);

// ============================================================ L D L^T
// Complex-symmetric factorisation without pivoting, S = L D L^T, for the
// FP32 + refinement solve of matrices with S = Z diag(s) symmetric: the
// PMCHWT matrix is [[A, -K], [K, C]] with A, C and K symmetric (the Galerkin
// L and K operators are), so Z diag(I, -I) = [[A, K], [K, -C]] is symmetric.
// Its diagonal blocks dominate enough that elimination without pivoting
// stays as accurate as partial pivoting on these systems (pivot growth below
// 5 at 2N = 960..3840); the refinement residual uses the original FP64 Z, and
// a factorisation that hits a zero pivot or does not let the refinement
// converge is redone with partial pivoting by the caller.  Half the flops of
// LU (the trailing update touches only the lower triangle) and no pivot
// search, so no grid-wide barrier per column.

// Exact (bitwise) symmetry tests of Z and of Z diag(I, -I), 32 x 32 tiles of
// the lower triangle against the mirrored tiles.  flags bit 0: Z is not
// symmetric; bit 1: Z diag(I, -I) is not (n odd counts as not).
__global__ void sym_check_kernel(const double2* __restrict__ Z, int64_t ldz, int n, unsigned* __restrict__ flags) {
    const int bi = blockIdx.y, bj = blockIdx.x;
    if (bj > bi) return;
    __shared__ double2 tt[32][33];
    __shared__ int done;
    if (threadIdx.x == 0) done = *(volatile unsigned*)flags == 3u;  // both tests already failed
    __syncthreads();
    if (done) return;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 256 threads
    const int half = (n % 2 == 0) ? n / 2 : -1;
    // tile (bj, bi) transposed into shared memory
    for (int r = ty; r < 32; r += 8) {
        const int i = bj * 32 + r, j = bi * 32 + tx;
        tt[r][tx] = (i < n && j < n) ? Z[(int64_t)i * ldz + j] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    unsigned bad = 0;
    for (int r = ty; r < 32; r += 8) {
        const int i = bi * 32 + r, j = bj * 32 + tx;
        if (i >= n || j >= n || j >= i) continue;
        const double2 a = Z[(int64_t)i * ldz + j];  // Z[i][j]
        const double2 b = tt[tx][r];                // Z[j][i]
        if (a.x != b.x || a.y != b.y) bad |= 1u;
        // (Z D)[i][j] = Z[i][j] s_j  vs  (Z D)[j][i] = Z[j][i] s_i
        const double si = (half >= 0 && i >= half) ? -1.0 : 1.0, sj = (half >= 0 && j >= half) ? -1.0 : 1.0;
        if (half < 0 || a.x * sj != b.x * si || a.y * sj != b.y * si) bad |= 2u;
    }
    bad = __reduce_or_sync(0xffffffffu, bad);
    if ((threadIdx.x & 31) == 0 && bad) atomicOr(flags, bad);
}

// Factors the jb x jb diagonal block at (j0, j0) in place: the strict lower
// triangle receives L, the diagonal D (the upper triangle is not touched).
// One CTA of 256 threads, thread i owning row i of the block.  The block is
// taken in 32-column sub-panels: each thread keeps its row's 32 sub-panel
// entries in registers and the columns are eliminated one at a time, with
// one block barrier per column (the pivot and the unscaled pivot column are
// published in shared memory, double-buffered by column parity); every row
// then scales by the pivot's reciprocal and applies the rank-1 update to
// its own registers.  The rest of the block's lower triangle is updated
// with the sub-panel: T = D L^T of the sub-panel is formed once in shared
// memory, and each thread accumulates an 8 x 4 set of outputs of a
// 128 x 64 block (rows ty + 16 r, columns tx + 16 c).  *info: first zero
// pivot (1-based).
constexpr int LDLT_SP = 32, LDLT_PITCH = LDLT_SP + 1, LDLT_TP = 256, LDLT_THREADS = 256;
constexpr size_t ldlt_smem_bytes(size_t esz) {
    return ((size_t)256 * LDLT_PITCH + (size_t)LDLT_SP * LDLT_TP) * esz;
}

template <typename R>
__global__ void __launch_bounds__(LDLT_THREADS, 1)
ldlt_diag_kernel(typename C2T<R>::type* __restrict__ A, int64_t lda, int j0, int jb, int* __restrict__ info) {
    using C2 = typename C2T<R>::type;
    extern __shared__ __align__(16) unsigned char ldlt_smem[];
    C2* P = reinterpret_cast<C2*>(ldlt_smem);  // [jb][LDLT_PITCH]: the eliminated sub-panel, rows c0..
    __shared__ C2 s_piv[2];                    // the pivot d of the column, by column parity
    __shared__ C2 s_col[2][LDLT_SP];           // unscaled column entries a[c][jj] of the sub-panel rows
    const int tid = threadIdx.x;
    C2 zero;
    zero.x = 0;
    zero.y = 0;
    for (int c0 = 0; c0 < jb; c0 += LDLT_SP) {
        const int w = min(LDLT_SP, jb - c0), rows = jb - c0;
        const int i = tid;  // this thread's row of the sub-panel
        const bool act = i < rows;
        // x[c] holds a[i][jj + c]: column jj is always x[0], the row shifting
        // left as columns retire (static register indices)
        C2 x[LDLT_SP];
#pragma unroll
        for (int c = 0; c < LDLT_SP; c++)
            x[c] = (act && c < w) ? A[(int64_t)(j0 + c0 + i) * lda + j0 + c0 + c] : zero;
        for (int jj = 0; jj < w; jj++) {
            const int par = jj & 1;
            if (i == jj) s_piv[par] = x[0];
            if (i > jj && i < w) s_col[par][i] = x[0];
            __syncthreads();
            const C2 d = s_piv[par];
            const bool zp = (d.x == 0 && d.y == 0);
            if (zp && i == jj) atomicCAS(info, 0, j0 + c0 + jj + 1);
            if (act && i > jj) {
                C2 one;
                one.x = 1;
                one.y = 0;
                const C2 inv = zp ? zero : cdiv(one, d);
                C2 l;
                l.x = x[0].x * inv.x - x[0].y * inv.y;
                l.y = x[0].x * inv.y + x[0].y * inv.x;
                // a[i][c] -= l_i (d l_c), d l_c being the unscaled a[c][jj]
#pragma unroll
                for (int c = 1; c < LDLT_SP; c++) {
                    if (jj + c < w) {
                        const C2 u = s_col[par][jj + c];
                        x[c].x -= l.x * u.x - l.y * u.y;
                        x[c].y -= l.x * u.y + l.y * u.x;
                    }
                }
                x[0] = l;
            }
            // column jj is final for this row: to shared memory, and its lower part to global
            if (act) {
                P[i * LDLT_PITCH + jj] = x[0];
                if (jj <= i) A[(int64_t)(j0 + c0 + i) * lda + j0 + c0 + jj] = x[0];
            }
#pragma unroll
            for (int c = 0; c + 1 < LDLT_SP; c++) x[c] = x[c + 1];
            x[LDLT_SP - 1] = zero;
        }
        __syncthreads();
        // the block's remaining lower triangle: A[i][c] -= sum_k L[i][k] d_k L[c][k]
        const int rest = rows - w;
        if (rest > 0) {
            C2* T = P + (size_t)256 * LDLT_PITCH;  // [k][c] = d_k L[w + c][k]
            for (int e = tid; e < w * rest; e += LDLT_THREADS) {
                const int k = e / rest, c = e % rest;
                const C2 dk = P[k * LDLT_PITCH + k], lc = P[(w + c) * LDLT_PITCH + k];
                C2 t;
                t.x = dk.x * lc.x - dk.y * lc.y;
                t.y = dk.x * lc.y + dk.y * lc.x;
                T[k * LDLT_TP + c] = t;
            }
            __syncthreads();
            // 128 x 64 output blocks of the lower triangle, 8 x 4 per thread
            const int ty = tid >> 4, tx = tid & 15, nbr = (rest + 127) / 128;
            for (int bi = 0; bi < nbr; bi++)
                for (int bc = 0; bc * 64 < min(rest, bi * 128 + 128); bc++) {
                    C2 acc[8][4];
                    int ii[8], cc[4];
#pragma unroll
                    for (int r = 0; r < 8; r++) ii[r] = bi * 128 + ty + 16 * r;
#pragma unroll
                    for (int c = 0; c < 4; c++) cc[c] = bc * 64 + tx + 16 * c;
#pragma unroll
                    for (int r = 0; r < 8; r++)
#pragma unroll
                        for (int c = 0; c < 4; c++)
                            acc[r][c] = (ii[r] < rest && cc[c] <= ii[r])
                                            ? A[(int64_t)(j0 + c0 + w + ii[r]) * lda + j0 + c0 + w + cc[c]]
                                            : zero;
#pragma unroll 2
                    for (int k = 0; k < w; k++) {
                        C2 a[8], b[4];
#pragma unroll
                        for (int r = 0; r < 8; r++) a[r] = ii[r] < rest ? P[(w + ii[r]) * LDLT_PITCH + k] : zero;
#pragma unroll
                        for (int c = 0; c < 4; c++) b[c] = T[k * LDLT_TP + cc[c]];
#pragma unroll
                        for (int r = 0; r < 8; r++)
#pragma unroll
                            for (int c = 0; c < 4; c++) {
                                acc[r][c].x -= a[r].x * b[c].x - a[r].y * b[c].y;
                                acc[r][c].y -= a[r].x * b[c].y + a[r].y * b[c].x;
                            }
                    }
#pragma unroll
                    for (int r = 0; r < 8; r++)
#pragma unroll
                        for (int c = 0; c < 4; c++)
                            if (ii[r] < rest && cc[c] <= ii[r])
                                A[(int64_t)(j0 + c0 + w + ii[r]) * lda + j0 + c0 + w + cc[c]] = acc[r][c];
                }
        }
        __syncthreads();
    }
}

// ------------------------------------- cluster L D L^T diagonal-block kernel
// The block of ldlt_diag_kernel (complex64) on one cluster of 8 CTAs, the
// block kept in distributed shared memory: CTA q holds block rows
// 32q..32q+31, columns 0..32q+31, so no entry makes a round trip through
// L2 between sub-panels.  Per 32-column sub-panel p:
//   A. CTA p factors the 32 x 32 diagonal sub-block with one warp (lane i:
//      row i, column by column), keeping the unscaled column entries in U;
//   cluster barrier;
//   B. every CTA q > p copies U and the pivots from CTA p and eliminates
//      the sub-panel columns of its own rows (one thread per row);
//   cluster barrier;
//   C. every CTA q > p updates its rows' lower triangle right of the
//      sub-panel: T = D L^T of block rows 32(p+1)..32q+31 is gathered from
//      CTAs p+1..q, then each thread accumulates 4 rows x 7 column groups.
// Every entry goes through the same operations, in the same order, as in
// ldlt_diag_kernel (the same pivot reciprocal, rank-1 updates in column
// order, T = d_k l_c, the trailing sums in k order).  2 np + 1 cluster
// barriers for np sub-panels, each at the top level of the kernel so that
// every thread of the cluster reaches it; no spin loop.  *info: first zero
// pivot (1-based).
constexpr int LDC_CTAS = 8, LDC_ROWS = 32, LDC_PITCH = 8 * LDC_ROWS + 1, LDC_UP = LDC_ROWS + 1,
              LDC_TP = 7 * LDC_ROWS + 1;
constexpr size_t ldlt_cluster_smem_bytes() {
    return ((size_t)LDC_ROWS * LDC_PITCH + 2 * (size_t)LDC_ROWS * LDC_UP + (size_t)LDC_ROWS * LDC_TP + 4 * LDC_ROWS) *
           sizeof(float2);
}

__global__ void __launch_bounds__(LDLT_THREADS, 1)
ldlt_diag_cluster_kernel(float2* __restrict__ A, int64_t lda, int j0, int jb, int* __restrict__ info) {
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    extern __shared__ __align__(16) unsigned char ldc_smem[];
    float2* S = reinterpret_cast<float2*>(ldc_smem);  // [32][LDC_PITCH]: this CTA's block rows
    float2* U = S + LDC_ROWS * LDC_PITCH;              // [32][LDC_UP]: unscaled sub-block entries (phase A)
    float2* UL = U + LDC_ROWS * LDC_UP;                // [32][LDC_UP]: CTA p's U (phase B)
    float2* T = UL + LDC_ROWS * LDC_UP;                // [32][LDC_TP]: d_k L[c][k] (phase C)
    float2* dk = T + LDC_ROWS * LDC_TP;                // [32]: the sub-panel's pivots
    float2* dinv = dk + LDC_ROWS;                      // [32]: their reciprocals (0 for a zero pivot)
    float2* s_col = dinv + LDC_ROWS;                   // [2][32]: column entries of phase A, by parity
    const int q = (int)cluster.block_rank(), tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int r0 = q * LDC_ROWS;                       // this CTA's first block row
    const int nr = max(0, min(LDC_ROWS, jb - r0));     // its rows inside the block
    const int ncol = min(r0 + LDC_ROWS, jb);           // columns kept: 0..ncol-1
    const float2 zero = make_float2(0.f, 0.f), one = make_float2(1.f, 0.f);
    // this CTA's rows, columns 0..ncol-1, eight independent loads in flight per thread
    const int nload = nr * ncol;
    for (int e0 = 0; e0 < nload; e0 += 8 * LDLT_THREADS) {
        float2 v[8];
#pragma unroll
        for (int u = 0; u < 8; u++) {
            const int e = e0 + u * LDLT_THREADS + tid;
            if (e < nload) v[u] = A[(int64_t)(j0 + r0 + e / ncol) * lda + j0 + e % ncol];
        }
#pragma unroll
        for (int u = 0; u < 8; u++) {
            const int e = e0 + u * LDLT_THREADS + tid;
            if (e < nload) S[(e / ncol) * LDC_PITCH + e % ncol] = v[u];
        }
    }
    __syncthreads();
    const int np = (jb + LDC_ROWS - 1) / LDC_ROWS;
    for (int p = 0; p < np; p++) {
        const int c0 = p * LDC_ROWS, w = min(LDC_ROWS, jb - c0);
        // A. the diagonal sub-block (rows c0.. of the block are this CTA's rows 0..w-1)
        if (q == p && wid == 0) {
            const int i = lane;
            const bool act = i < w;
            float2 x[LDC_ROWS];  // x[c] = a[i][jj + c], shifted left as columns retire
#pragma unroll
            for (int c = 0; c < LDC_ROWS; c++) x[c] = (act && c < w) ? S[i * LDC_PITCH + c0 + c] : zero;
            for (int jj = 0; jj < w; jj++) {
                const int par = jj & 1;
                if (act) s_col[par * LDC_ROWS + i] = x[0];
                __syncwarp();
                const float2 d = s_col[par * LDC_ROWS + jj];
                const bool zp = (d.x == 0 && d.y == 0);
                if (zp && i == jj) atomicCAS(info, 0, j0 + c0 + jj + 1);
                if (act && i > jj) {
                    const float2 inv = zp ? zero : cdiv(one, d);
                    float2 l;
                    l.x = x[0].x * inv.x - x[0].y * inv.y;
                    l.y = x[0].x * inv.y + x[0].y * inv.x;
#pragma unroll
                    for (int c = 1; c < LDC_ROWS; c++) {
                        if (jj + c < w) {
                            const float2 u = s_col[par * LDC_ROWS + jj + c];
                            x[c].x -= l.x * u.x - l.y * u.y;
                            x[c].y -= l.x * u.y + l.y * u.x;
                        }
                    }
                    U[i * LDC_UP + jj] = x[0];
                    x[0] = l;
                }
                if (act && jj <= i) S[i * LDC_PITCH + c0 + jj] = x[0];
#pragma unroll
                for (int c = 0; c + 1 < LDC_ROWS; c++) x[c] = x[c + 1];
                x[LDC_ROWS - 1] = zero;
            }
        }
        cluster.sync();
        // B. this CTA's rows below the sub-block
        if (q > p && nr > 0) {
            const float2* Up = cluster.map_shared_rank(U, p);
            const float2* Sp = cluster.map_shared_rank(S, p);
            for (int e = tid; e < w * w; e += LDLT_THREADS) {
                const int r = e / w, c = e % w;
                if (c < r) UL[r * LDC_UP + c] = Up[r * LDC_UP + c];
            }
            if (tid < w) {
                const float2 d = Sp[tid * LDC_PITCH + c0 + tid];
                dk[tid] = d;
                dinv[tid] = (d.x == 0 && d.y == 0) ? zero : cdiv(one, d);
            }
            __syncthreads();
            if (wid == 0 && lane < nr) {
                const int i = lane;
                float2 x[LDC_ROWS];
#pragma unroll
                for (int c = 0; c < LDC_ROWS; c++) x[c] = c < w ? S[i * LDC_PITCH + c0 + c] : zero;
                for (int jj = 0; jj < w; jj++) {
                    const float2 inv = dinv[jj];
                    float2 l;
                    l.x = x[0].x * inv.x - x[0].y * inv.y;
                    l.y = x[0].x * inv.y + x[0].y * inv.x;
#pragma unroll
                    for (int c = 1; c < LDC_ROWS; c++) {
                        if (jj + c < w) {
                            const float2 u = UL[(jj + c) * LDC_UP + jj];
                            x[c].x -= l.x * u.x - l.y * u.y;
                            x[c].y -= l.x * u.y + l.y * u.x;
                        }
                    }
                    S[i * LDC_PITCH + c0 + jj] = l;
#pragma unroll
                    for (int c = 0; c + 1 < LDC_ROWS; c++) x[c] = x[c + 1];
                    x[LDC_ROWS - 1] = zero;
                }
            }
        }
        cluster.sync();
        // C. this CTA's rows, columns cs..r0+31 of the lower triangle
        if (q > p && nr > 0) {
            const int cs = c0 + w, nc = r0 + LDC_ROWS - cs, ng = nc / 32;  // ng = q - p <= 7
            // four independent remote loads in flight per thread
            for (int e0 = 0; e0 < w * nc; e0 += 4 * LDLT_THREADS) {
                float2 lc[4];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const int e = e0 + u * LDLT_THREADS + tid, c = e / w, k = e % w, row = cs + c;
                    lc[u] = zero;
                    if (e < w * nc && row < jb)
                        lc[u] = cluster.map_shared_rank(S, row / LDC_ROWS)[(row % LDC_ROWS) * LDC_PITCH + c0 + k];
                }
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const int e = e0 + u * LDLT_THREADS + tid, c = e / w, k = e % w;
                    if (e < w * nc) {
                        const float2 d = dk[k];
                        float2 t;
                        t.x = d.x * lc[u].x - d.y * lc[u].y;
                        t.y = d.x * lc[u].y + d.y * lc[u].x;
                        T[k * LDC_TP + c] = t;
                    }
                }
            }
            __syncthreads();
            float2 acc[4][7];
            bool ok[4][7];
#pragma unroll
            for (int r = 0; r < 4; r++)
#pragma unroll
                for (int g = 0; g < 7; g++) {
                    const int i = wid * 4 + r, col = cs + lane + 32 * g;
                    ok[r][g] = g < ng && i < nr && col <= r0 + i;
                    acc[r][g] = ok[r][g] ? S[i * LDC_PITCH + col] : zero;
                }
#pragma unroll 2
            for (int k = 0; k < w; k++) {
                float2 a[4];
#pragma unroll
                for (int r = 0; r < 4; r++) a[r] = S[(wid * 4 + r) * LDC_PITCH + c0 + k];
#pragma unroll
                for (int g = 0; g < 7; g++)
                    if (g < ng) {  // the column groups this CTA has at this sub-panel
                        const float2 b = T[k * LDC_TP + lane + 32 * g];
#pragma unroll
                        for (int r = 0; r < 4; r++) {
                            acc[r][g].x -= a[r].x * b.x - a[r].y * b.y;
                            acc[r][g].y -= a[r].x * b.y + a[r].y * b.x;
                        }
                    }
            }
#pragma unroll
            for (int r = 0; r < 4; r++)
#pragma unroll
                for (int g = 0; g < 7; g++)
                    if (ok[r][g]) S[(wid * 4 + r) * LDC_PITCH + cs + lane + 32 * g] = acc[r][g];
            __syncthreads();
        }
    }
    __syncthreads();
    for (int r = wid; r < nr; r += LDLT_THREADS / 32)
        for (int c = lane; c <= r0 + r; c += 32) A[(int64_t)(j0 + r0 + r) * lda + j0 + c] = S[r * LDC_PITCH + c];
    // no CTA leaves while another may still read its shared memory
    cluster.sync();
}

// Whether the cluster diagonal-block kernel can be resident on this device
// (8 CTAs with its shared memory; asked once per device and remembered).
static bool ldlt_cluster_fits(bem_ctx* ctx) {
    static std::mutex mu;
    static std::map<int, bool> ok;
    std::lock_guard<std::mutex> lk(mu);
    auto it = ok.find(ctx->device);
    if (it != ok.end()) return it->second;
    bool fits = cudaFuncSetAttribute(ldlt_diag_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)ldlt_cluster_smem_bytes()) == cudaSuccess;
    if (fits) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(LDC_CTAS);
        cfg.blockDim = dim3(LDLT_THREADS);
        cfg.dynamicSmemBytes = ldlt_cluster_smem_bytes();
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = LDC_CTAS;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int ncl = 0;
        fits = cudaOccupancyMaxActiveClusters(&ncl, (const void*)ldlt_diag_cluster_kernel, &cfg) == cudaSuccess &&
               ncl >= 1;
    }
    if (!fits) cudaGetLastError();
    ok[ctx->device] = fits;
    return fits;
}

static int launch_ldlt_diag_cluster(bem_ctx* ctx, float2* A, int64_t lda, int j0, int jb, int* d_info) {
    if (jb < 1 || jb > LDC_CTAS * LDC_ROWS) return fail(ctx, BEM_ERR_INVALID, "cluster diagonal block: jb out of range");
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(LDC_CTAS);
    cfg.blockDim = dim3(LDLT_THREADS);
    cfg.dynamicSmemBytes = ldlt_cluster_smem_bytes();
    cfg.stream = ctx->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = LDC_CTAS;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    BEM_TRY_CUDA(ctx, cudaLaunchKernelEx(&cfg, ldlt_diag_cluster_kernel, A, lda, j0, jb, d_info));
    BEM_LAUNCHED(ctx);
    return BEM_OK;
}

int sym_structure(bem_ctx* ctx, const double2* Z, int64_t ldz, int n, bool* sym, bool* sym_half) {
    unsigned* d_flags = nullptr;
    BEM_TRY_CUDA(ctx, cudaMalloc(&d_flags, sizeof(unsigned)));
    int s = BEM_OK;
    unsigned h = 3;
    do {
        if (cudaMemsetAsync(d_flags, 0, sizeof(unsigned), ctx->stream) != cudaSuccess) {
            s = fail(ctx, BEM_ERR_CUDA, "symmetry check");
            break;
        }
        const int T = (n + 31) / 32;
        if (T > 65535) {
            s = fail(ctx, BEM_ERR_INVALID, "symmetry check: n too large");
            break;
        }
        sym_check_kernel<<<dim3(T, T), 256, 0, ctx->stream>>>(Z, ldz, n, d_flags);
        ctx->launches++;
        if (cudaMemcpyAsync(&h, d_flags, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
            cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
            s = fail(ctx, BEM_ERR_CUDA, "symmetry check: %s", cudaGetErrorString(cudaGetLastError()));
            break;
        }
    } while (0);
    cudaFree(d_flags);
    *sym = s == BEM_OK && !(h & 1u);
    *sym_half = s == BEM_OK && !(h & 2u);
    return s;
}

// W[c][r] (column-major, ld 256) = -1 on the diagonal, 0 elsewhere.
__global__ void neg_eye_kernel(float2* __restrict__ W, int jb) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= jb * TRSM_KB) return;
    const int c = t / TRSM_KB, r = t % TRSM_KB;
    W[t] = make_float2(r == c ? -1.f : 0.f, 0.f);
}

// Blocked right-looking L D L^T of the row-major complex64 S (lower triangle).
// Per 256-column block: the diagonal block is factored in one CTA; its
// inverse factor W = L11^-T D^-1 comes from a block TRSM on -I; the panel
// below becomes L21 = S21 W in one tensor-core GEMM (in place: the operands
// are packed before the product is written); then the lower-triangle update.
// L[c * 256 + r] = W[c * 256 + r] d_r for r, c < jb (W = -L11^-1 D^-1 of the
// diagonal block at j0, d_r its pivots), 0 elsewhere: -L11^-1 itself.
__global__ void linv_from_w_kernel(const float2* __restrict__ W, const float2* __restrict__ A, int64_t lda, int j0,
                                   int jb, float2* __restrict__ L) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= TRSM_KB * TRSM_KB) return;
    const int c = t / TRSM_KB, r = t % TRSM_KB;
    float2 v = make_float2(0.f, 0.f);
    if (r < jb && c < jb) {
        const float2 w = W[t], d = A[(int64_t)(j0 + r) * lda + j0 + r];
        v = make_float2(w.x * d.x - w.y * d.y, w.x * d.y + w.y * d.x);
    }
    L[t] = v;
}

int sytrf_nopiv(bem_ctx* ctx, float2* A, int64_t lda, int n, int* d_info, float2* Linv) {
    using C2 = float2;
    const int NB = TRSM_KB;
    const size_t smem = ldlt_smem_bytes(sizeof(C2));
    static_assert(ldlt_smem_bytes(sizeof(float2)) <= 227 * 1024, "L D L^T diagonal block shared memory");
    BEM_TRY_CUDA(ctx, cudaFuncSetAttribute(ldlt_diag_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem));
    // the diagonal blocks on one 8-CTA cluster where it fits, else on one CTA
    const bool diag_cluster = ctx->ldlt_cluster && ldlt_cluster_fits(ctx);
    BEM_TRY_CUDA(ctx, cudaMemsetAsync(d_info, 0, sizeof(int), ctx->stream));
    BEM_TRY_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream));
    struct Buf {
        float2* p = nullptr;
        ~Buf() {
            if (p) cudaFree(p);
        }
    } W;
    BEM_TRY_CUDA(ctx, cudaMalloc(&W.p, (size_t)NB * NB * sizeof(float2)));
    // the diagonal block at j0 and its panel below: L D L^T of the block,
    // then L21 = S21 L11^-T D^-1 for the rows [j0 + jb, n)
    auto factor_block = [&](int j0, int jb) -> int {
        const int below = n - j0 - jb;
        cudaEvent_t ev = ctx->prof_begin(PROF_PANEL);
        if (diag_cluster) {
            BEM_TRY(launch_ldlt_diag_cluster(ctx, A, lda, j0, jb, d_info));
        } else {
            ldlt_diag_kernel<float><<<1, LDLT_THREADS, smem, ctx->stream>>>(A, lda, j0, jb, d_info);
            BEM_LAUNCHED(ctx);
        }
        if (ev) ctx->prof_end(PROF_PANEL, ev, 8.0 * jb * (double)jb * jb / 3, 16.0 * (double)jb * jb);
        if (below > 0 || Linv) {
            // column c of W.p solves L11 x = -e_c, then x_r /= d_r:
            // W.p[c * 256 + r] = -L11^-1[r][c] / d_r
            neg_eye_kernel<<<(jb * NB + 255) / 256, 256, 0, ctx->stream>>>(W.p, jb);
            BEM_LAUNCHED(ctx);
            BEM_TRY((trsm_block<float, false, false, TRSM_DIVDIAG>(ctx, A, lda, j0, jb, W.p, NB, 0, jb, 0)));
        }
        if (Linv) {
            linv_from_w_kernel<<<NB * NB / 256, 256, 0, ctx->stream>>>(W.p, A, lda, j0, jb,
                                                                     Linv + (size_t)(j0 / NB) * NB * NB);
            BEM_LAUNCHED(ctx);
        }
        if (below > 0) {
            // L21 = S21 L11^-T D^-1: B given row-major (K x N) is
            // B[k][j] = W.p[k * 256 + j] = -(L11^-T D^-1)[k][j]; the store mode writes C = -A B
            TcOpts o;
            o.b_rowmajor = true;
            o.store = true;
            o.prof_cls = PROF_PANEL_UPDATE;
            float2* S21 = A + (int64_t)(j0 + jb) * lda + j0;
            BEM_TRY(tc_gemm_ex(ctx, below, jb, jb, S21, lda, W.p, NB, S21, lda, o));
        }
        return (int)BEM_OK;
    };
    // Super-blocks of factor_sb 256-column blocks: each block is factored and
    // updates the super-block's later block columns alone (thin GEMMs), and
    // the lower-triangle update of the rest takes the whole super-block
    // (K = 256 factor_sb: fewer launches and fewer read-modify-writes of the
    // trailing matrix).
    const int SB = std::max(1, std::min(4, ctx->factor_sb)) * NB;
    for (int J0 = 0; J0 < n; J0 += SB) {
        const int JB = std::min(SB, n - J0);
        for (int j = J0; j < J0 + JB; j += NB) {
            const int jb = std::min(NB, J0 + JB - j);
            BEM_TRY(factor_block(j, jb));
            const int nc = J0 + JB - j - jb;  // the super-block's columns after this block
            if (nc > 0) {
                // S[j+jb:, j+jb:J0+JB] -= L21 D L21^T (rows j+jb.. of this block's L21)
                TcOpts o;
                o.bscale = A + (int64_t)j * lda + j;
                o.bscale_stride = lda + 1;
                o.prof_cls = PROF_LU_UPDATE;
                const float2* L21 = A + (int64_t)(j + jb) * lda + j;
                BEM_TRY(tc_gemm_ex(ctx, n - j - jb, nc, jb, L21, lda, L21, lda, A + (int64_t)(j + jb) * lda + j + jb,
                                   lda, o));
            }
        }
        const int below = n - J0 - JB;
        if (below > 0) {
            // S22 -= L21 D L21^T over the super-block, lower triangle
            TcOpts o;
            o.lower = true;
            o.bscale = A + (int64_t)J0 * lda + J0;
            o.bscale_stride = lda + 1;
            o.prof_cls = PROF_LU_UPDATE;
            const float2* L21 = A + (int64_t)(J0 + JB) * lda + J0;
            BEM_TRY(tc_gemm_ex(ctx, below, below, JB, L21, lda, L21, lda, A + (int64_t)(J0 + JB) * lda + J0 + JB, lda,
                               o));
        }
    }
    return BEM_OK;
}

// X[i][c] /= D_i
__global__ void diag_div_kernel(const float2* __restrict__ A, int64_t lda, float2* __restrict__ X, int64_t ldx, int n,
                                int nrhs) {
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)n * nrhs) return;
    const int r = (int)(t % n), c = (int)(t / n);
    X[(int64_t)c * ldx + r] = cdiv(X[(int64_t)c * ldx + r], A[(int64_t)r * lda + r]);
}

// X = S^-1 B with S = L D L^T (B, X column-major complex64; X may alias B).
int sytrs_nopiv(bem_ctx* ctx, const float2* A, int64_t lda, int n, const float2* B, int64_t ldb, float2* X,
                int64_t ldx, int nrhs, const float2* Linv, float2* tmp) {
    const int NB = TRSM_KB;
    if (nrhs <= 0) return BEM_OK;
    int64_t tot = (int64_t)n * nrhs;
    if (B != X || ldb != ldx) {
        permute_rows_kernel<float><<<(unsigned)((tot + 255) / 256), 256, 0, ctx->stream>>>(B, ldb, X, ldx, nullptr, n,
                                                                                         nrhs);
        BEM_LAUNCHED(ctx);
    }
    // Super-blocks of solve_sb 256-row diagonal blocks: the blocks of a
    // super-block update one another with thin GEMMs, so the update of all
    // rows beyond runs with K = 256 solve_sb (fewer launches and fewer
    // read-modify-writes of X).
    const int SB = std::max(1, std::min(4, ctx->solve_sb)) * NB;
    auto update = [&](int M, int K, const float2* Ablk, bool trans, float2* Bx, float2* Cx) {
        TcOpts o;
        o.c_colmajor = true;
        o.a_trans = trans;
        o.prof_cls = PROF_SOLVE_UPDATE;
        return tc_gemm_ex(ctx, M, nrhs, K, Ablk, lda, Bx, ldx, Cx, ldx, o);
    };
    // the diagonal block at J0 (jb rows): X_blk = L11^-1 X_blk (back: L11^-T),
    // as -(-L11^-1) tmp with tmp a copy of X_blk, or a block triangular solve
    auto diag = [&](int J0, int jb, bool back) -> int {
        if (!Linv || !tmp) {
            if (back)
                return trsm_block<float, true, false, TRSM_TRANS | TRSM_UNIT>(ctx, A, lda, J0, jb, X, ldx, 0, nrhs);
            return trsm_block<float, false, false>(ctx, A, lda, J0, jb, X, ldx, 0, nrhs);
        }
        BEM_TRY_CUDA(ctx, cudaMemcpy2DAsync(tmp, NB * sizeof(float2), X + J0, ldx * sizeof(float2),
                                            jb * sizeof(float2), nrhs, cudaMemcpyDeviceToDevice, ctx->stream));
        TcOpts o;
        o.c_colmajor = true;
        o.store = true;
        o.a_trans = !back;  // forward: A[r][c] = Li[c * 256 + r]; back: A[r][c] = Li[r * 256 + c]
        o.prof_cls = PROF_TRSM;
        const float2* Li = Linv + (size_t)(J0 / NB) * NB * NB;
        return tc_gemm_ex(ctx, jb, nrhs, jb, Li, NB, tmp, NB, X + J0, ldx, o);
    };
    // L z = b
    for (int J0 = 0; J0 < n; J0 += SB) {
        const int JB = std::min(SB, n - J0);
        for (int j = J0; j < J0 + JB; j += NB) {
            const int jb = std::min(NB, J0 + JB - j), nc = J0 + JB - j - jb;
            BEM_TRY(diag(j, jb, false));
            // the super-block's later rows: X[j+jb:J0+JB] -= L[j+jb:J0+JB, j:j+jb] X[j:j+jb]
            if (nc > 0) BEM_TRY(update(nc, jb, A + (int64_t)(j + jb) * lda + j, false, X + j, X + j + jb));
        }
        const int below = n - J0 - JB;
        if (below > 0) BEM_TRY(update(below, JB, A + (int64_t)(J0 + JB) * lda + J0, false, X + J0, X + J0 + JB));
    }
    // y = D^-1 z
    diag_div_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, ctx->stream>>>(A, lda, X, ldx, n, nrhs);
    BEM_LAUNCHED(ctx);
    // L^T x = y, super-blocks from the last
    const int nsb = (n + SB - 1) / SB;
    for (int bi = nsb - 1; bi >= 0; bi--) {
        const int J0 = bi * SB, JB = std::min(SB, n - J0);
        for (int j = J0 + ((JB - 1) / NB) * NB; j >= J0; j -= NB) {
            const int jb = std::min(NB, J0 + JB - j);
            BEM_TRY(diag(j, jb, true));
            // the super-block's earlier rows: X[J0:j] -= (L[j:j+jb, J0:j])^T X[j:j+jb]
            if (j > J0) BEM_TRY(update(j - J0, jb, A + (int64_t)j * lda + J0, true, X + j, X + J0));
        }
        // X[0:J0] -= (L[J0:J0+JB, 0:J0])^T X[J0:J0+JB]
        if (J0 > 0) BEM_TRY(update(J0, JB, A + (int64_t)J0 * lda, true, X + J0, X));
    }
    return BEM_OK;
}

// Row pivots (LAPACK interchange sequence, 0-based) -> gather permutation.
void pivots_to_perm(const std::vector<int>& ipiv, std::vector<int>& perm) {
    int n = (int)ipiv.size();
    perm.resize(n);
    for (int i = 0; i < n; i++) perm[i] = i;
    for (int k = 0; k < n; k++) std::swap(perm[k], perm[ipiv[k]]);
}

}  // namespace bem
