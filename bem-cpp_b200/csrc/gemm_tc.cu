// Three-product complex GEMM on the fifth-generation tensor cores (tcgen05 +
// TMA + TMEM), used for the big updates of the FP32 factorisation and solves:
//
//   C -= A * B      A: M x K complex (K contiguous), B: K x N complex,
//                   C: M x N complex64, row-major (LU) or column-major (solves)
//
// The complex product is written as one real GEMM over interleaved columns:
//   C'[i, 2j+{0,1}] -= sum_k' A'[i, k'] B'[2j+{0,1}, k']
// with A'[i, 2k] = Re a_ik, A'[i, 2k+1] = Im a_ik (the raw float layout of a
// complex row) and B' rows (Re b, -Im b) / (Im b, Re b) interleaved over k.
// Every operand is split x = hi + lo and the product taken as
// hi*hi + hi*lo + lo*hi, accumulated in FP32 in TMEM.  Two splits:
//  * FP16 parts (context option tensor_split = 1, the default; kind::f16 at
//    twice the TF32 rate): each row of A' and each complex column of B is
//    first scaled by a power of two that brings its largest part into
//    [2^14, 2^15), so no part overflows FP16, and the parts of small entries
//    that fall below FP16's normal range lose at most 2^-38 of the row's
//    largest entry; the epilogue multiplies the accumulator by the inverse
//    scales of its row and column (exact: powers of two).
//  * TF32 parts (tensor_split = 0; kind::tf32): hi, lo rounded to TF32.
//
// Pack kernels write the hi / lo operands K-major.  Both GEMM kernels stream
// 128-row A and 256-row B tiles of one 128-byte swizzle row of K per stage
// (32 floats or 64 halves) with TMA (no multicast) through a 2-stage mbarrier
// pipeline: a stage holds hi and lo of both tiles, 96 KB, so two fill the
// shared memory.  One thread issues tcgen05.mma (M = 128, N = 256; K = 8 for
// TF32, 16 for FP16) into a 128 x 256 FP32 TMEM accumulator.
//  * gemm_kernel: one CTA per output tile; four warps read the accumulator
//    back with tcgen05.ld and apply C -= acc.
//  * gemm_persistent_kernel (default): one CTA per SM walking the tiles in
//    grouped raster order, warp-specialised (warp 0 TMA producer, warp 1 MMA
//    issuer, warps 2-5 epilogue) with two TMEM accumulators (512 columns) so
//    the epilogue of one tile overlaps the MMAs of the next.
// Every wait is bounded (~1 s of clock cycles): on expiry the kernel records
// BEM_ERR_TIMEOUT in the status word, drains the copies it issued, frees its
// TMEM and returns.
#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdint>
#include <cstring>

#include "bem_internal.h"
#include "lu_internal.h"

namespace bem {

namespace tc {

constexpr int BM = 128;       // rows per tile
constexpr int BN = 256;       // real columns per tile (128 complex)
constexpr int BK = 32;        // floats of K per stage (one 128-byte swizzle row)
constexpr int STAGES = 2;
constexpr int A_BYTES = BM * BK * 4;   // 16 KB
constexpr int B_BYTES = BN * BK * 4;   // 32 KB
constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;  // hi + lo of each: 96 KB
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 /*align*/ + 256 /*barriers*/;
constexpr uint32_t TMEM_COLS = 256;
constexpr long long WAIT_CYCLES = 2000000000LL;  // ~1 s at 2 GHz

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait on an mbarrier phase; false (and the status word set) on expiry
// or when another thread of the CTA already gave up.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int* status, volatile int* abort_flag) {
    long long t0 = clock64();
    while (!mbar_try(bar, parity)) {
        if (*abort_flag) return false;
        if (clock64() - t0 > WAIT_CYCLES) {
            atomicCAS(status, 0, (int)BEM_ERR_TIMEOUT);
            *abort_flag = 1;
            return false;
        }
    }
    return true;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

// K-major operand tile with 128-byte swizzle: rows of 128 B, 8-row groups
// 1024 B apart (SBO), LBO unused (1), descriptor version 1.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;                 // leading byte offset (16 B units), unused for SW128 K-major
    d |= (uint64_t)(1024 >> 4) << 32;       // stride byte offset: 8 rows x 128 B
    d |= (uint64_t)1 << 46;                 // descriptor version (Blackwell)
    d |= (uint64_t)2 << 61;                 // layout: SWIZZLE_128B
    return d;
}

// kind::tf32, FP32 accumulate, A and B K-major, M = 128, N = 256.
constexpr uint32_t IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(BN >> 3) << 17) |
                           ((uint32_t)(BM >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t accumulate) {
    uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        ::"r"(tmem_d), "l"(a), "l"(b), "r"(IDESC), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
}

// kind::f16 with FP16 A and B (both the same type), FP32 accumulate, K-major,
// M = 128, N = 256; one MMA covers K = 16 halves = 32 bytes of a swizzle row,
// the same byte step as K = 8 of kind::tf32.
constexpr uint32_t IDESC_F16 = (1u << 4) | (0u << 7) | (0u << 10) | ((uint32_t)(BN >> 3) << 17) |
                               ((uint32_t)(BM >> 4) << 24);

__device__ __forceinline__ void mma_f16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t accumulate) {
    uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        ::"r"(tmem_d), "l"(a), "l"(b), "r"(IDESC_F16), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
          "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
          "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
          "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ float to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// C (complex64) -= A' B'^T over one 128 x 256 tile.  c_colmajor: C[j*ldc + i].
__global__ void __launch_bounds__(128, 1)
gemm_kernel(const __grid_constant__ CUtensorMap tA_hi, const __grid_constant__ CUtensorMap tA_lo,
            const __grid_constant__ CUtensorMap tB_hi, const __grid_constant__ CUtensorMap tB_lo,
            float2* __restrict__ C, int64_t ldc, int c_colmajor, int M, int Nc, int K2, int* status) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t* bars = (uint64_t*)(smem + STAGES * STAGE_BYTES);  // full[S], empty[S], accum
    uint32_t* tmem_slot = (uint32_t*)(bars + 2 * STAGES + 1);
    __shared__ volatile int abort_flag;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int nk = (K2 + BK - 1) / BK;

    if (threadIdx.x == 0) {
        abort_flag = 0;
        for (int s = 0; s < STAGES; s++) {
            mbar_init(smem_u32(&bars[s]), 1);
            mbar_init(smem_u32(&bars[STAGES + s]), 1);
        }
        mbar_init(smem_u32(&bars[2 * STAGES]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (threadIdx.x == 0) {
        // TMA producer
        for (int kt = 0; kt < nk; kt++) {
            const int s = kt % STAGES;
            if (kt >= STAGES && !mbar_wait(smem_u32(&bars[STAGES + s]), ((kt / STAGES) - 1) & 1, status, &abort_flag))
                break;
            unsigned char* st = smem + s * STAGE_BYTES;
            const uint32_t full = smem_u32(&bars[s]);
            mbar_expect_tx(full, STAGE_BYTES);
            tma_load_2d(smem_u32(st), &tA_hi, kt * BK, m0, full);
            tma_load_2d(smem_u32(st + A_BYTES), &tA_lo, kt * BK, m0, full);
            tma_load_2d(smem_u32(st + 2 * A_BYTES), &tB_hi, kt * BK, n0, full);
            tma_load_2d(smem_u32(st + 2 * A_BYTES + B_BYTES), &tB_lo, kt * BK, n0, full);
        }
    } else if (threadIdx.x == 32) {
        // MMA issuer
        bool ok = true;
        for (int kt = 0; kt < nk && ok; kt++) {
            const int s = kt % STAGES;
            if (!mbar_wait(smem_u32(&bars[s]), (kt / STAGES) & 1, status, &abort_flag)) {
                ok = false;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            unsigned char* st = smem + s * STAGE_BYTES;
            const uint32_t a_hi = smem_u32(st), a_lo = smem_u32(st + A_BYTES);
            const uint32_t b_hi = smem_u32(st + 2 * A_BYTES), b_lo = smem_u32(st + 2 * A_BYTES + B_BYTES);
#pragma unroll
            for (int ks = 0; ks < BK / 8; ks++) {
                // advance 8 floats (32 B) along K inside the swizzle row
                const uint32_t off = ks * 32;
                const uint64_t dah = smem_desc(a_hi + off), dal = smem_desc(a_lo + off);
                const uint64_t dbh = smem_desc(b_hi + off), dbl = smem_desc(b_lo + off);
                mma_tf32(tmem, dah, dbh, (kt > 0 || ks > 0) ? 1u : 0u);
                mma_tf32(tmem, dah, dbl, 1u);
                mma_tf32(tmem, dal, dbh, 1u);
            }
            mma_commit(smem_u32(&bars[STAGES + s]));  // stage s free once these MMAs read it
        }
        mma_commit(smem_u32(&bars[2 * STAGES]));      // accumulator ready
    }
    __syncwarp();

    // epilogue: 4 warps x 32 TMEM lanes = 128 rows
    bool ok = mbar_wait(smem_u32(&bars[2 * STAGES]), 0, status, &abort_flag);
    ok = __all_sync(0xffffffffu, ok);
    if (ok) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int row = m0 + warp * 32 + lane;
        const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
        for (int ch = 0; ch < BN / 32; ch++) {
            float v[32];
            tmem_ld32(lane_base + ch * 32, v);
            if (row < M) {
                const int c0 = (n0 >> 1) + ch * 16;
#pragma unroll
                for (int j = 0; j < 16; j++) {
                    const int col = c0 + j;
                    if (col < Nc) {
                        float2* p = c_colmajor ? &C[(int64_t)col * ldc + row] : &C[(int64_t)row * ldc + col];
                        float2 c = *p;
                        c.x -= v[2 * j];
                        c.y -= v[2 * j + 1];
                        *p = c;
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
    }
}

// Persistent, warp-specialised version: one CTA per SM walks a grouped
// raster of 128 x 256 tiles.  Warp 0 issues TMA, warp 1 issues tcgen05.mma
// into one of two 256-column TMEM accumulators, warps 2-5 drain the other
// accumulator into C, so the read-modify-write of tile i overlaps the MMAs of
// tile i+1.  Barriers: full/empty per smem stage, tfull/tempty per
// accumulator (tempty counts the four epilogue warps).
// Raster: groups of gm row tiles x all column tiles (gm = 16 by default,
// bem_ctx_set_option "gemm_group_m"); a wave of 148 tiles then spans ~16 row x
// ~9 column tiles (8 MB of A and 9 MB of B panels in L2 at K = 256), which
// halves the B-panel re-reads against groups of 8.
constexpr uint32_t TMEM_COLS2 = 512;

struct TileMap {
    int num_m, num_n;
    int gm;     // row tiles per raster group
    int lower;  // square C, only tiles on or below the diagonal (BM rows == BN / 2 complex columns)
    __device__ __forceinline__ int count() const {
        return lower ? num_m * (num_m + 1) / 2 : num_m * num_n;
    }
    // Grouped raster: gm row tiles at a time, column by column.  For the
    // lower triangle only the tiles on or below the diagonal are enumerated
    // (row group g starts at tile S(g) = G g (G g + 1) / 2), so consecutive
    // CTAs stay on neighbouring tiles and share their operand panels in L2.
    __device__ __forceinline__ void tile(int t, int& mt, int& nt) const {
        if (!lower) {
            const int per_group = gm * num_n;
            const int g = t / per_group, first_m = g * gm;
            const int gsize = min(gm, num_m - first_m);
            const int r = t % per_group;
            mt = first_m + r % gsize;
            nt = r / gsize;
            return;
        }
        // largest y with y (y + 1) / 2 <= t, then the group of row y
        long long y = (long long)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
        while (y > 0 && y * (y + 1) / 2 > t) y--;
        while ((y + 1) * (y + 2) / 2 <= t) y++;
        const int g = (int)(y / gm), first_m = g * gm;
        const int gsize = min(gm, num_m - first_m);
        int r = t - (int)((long long)first_m * (first_m + 1) / 2);
        if (r < gsize * first_m) {  // columns left of the group's diagonal block
            nt = r / gsize;
            mt = first_m + r % gsize;
            return;
        }
        r -= gsize * first_m;
        for (int c = 0; c < gsize; c++) {  // the diagonal block, column by column
            if (r < gsize - c) {
                nt = first_m + c;
                mt = first_m + c + r;
                return;
            }
            r -= gsize - c;
        }
        mt = nt = num_m - 1;  // not reached for t < count()
    }
    __device__ __forceinline__ bool skip(int, int) const { return false; }
};

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// F16: operand parts are FP16 (kind::f16, 64 halves per 128-byte stage row)
// and sa / sb hold the (scale, inverse) pairs of the rows of A' and the
// complex columns of B; else TF32 parts (kind::tf32, 32 floats per row).
template <bool F16>
__global__ void __launch_bounds__(192, 1)
gemm_persistent_kernel(const __grid_constant__ CUtensorMap tA_hi, const __grid_constant__ CUtensorMap tA_lo,
                       const __grid_constant__ CUtensorMap tB_hi, const __grid_constant__ CUtensorMap tB_lo,
                       float2* __restrict__ C, int64_t ldc, int c_colmajor, int M, int Nc, int K2, int lower,
                       int store, int group_m, int* status, const float2* __restrict__ sa,
                       const float2* __restrict__ sb) {
    constexpr int BKE = F16 ? 2 * BK : BK;  // elements of K per stage (one 128-byte row)
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t* bars = (uint64_t*)(smem + STAGES * STAGE_BYTES);
    uint64_t* full = bars;                  // [STAGES]
    uint64_t* empty = bars + STAGES;        // [STAGES]
    uint64_t* tfull = bars + 2 * STAGES;    // [2]
    uint64_t* tempty = bars + 2 * STAGES + 2;
    uint32_t* tmem_slot = (uint32_t*)(bars + 2 * STAGES + 4);
    __shared__ volatile int abort_flag;
    __shared__ int issued_total, consumed_total;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nk = (K2 + BKE - 1) / BKE;
    TileMap tm;
    tm.num_m = (M + BM - 1) / BM;
    tm.num_n = (2 * Nc + BN - 1) / BN;
    tm.lower = lower;
    tm.gm = group_m > 0 ? group_m : 16;
    const int ntiles = tm.count();

    if (threadIdx.x == 0) {
        abort_flag = 0;
        issued_total = consumed_total = 0;
        for (int s = 0; s < STAGES; s++) {
            mbar_init(smem_u32(&full[s]), 1);
            mbar_init(smem_u32(&empty[s]), 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(smem_u32(&tfull[b]), 1);
            mbar_init(smem_u32(&tempty[b]), 4);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TMEM_COLS2));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            int it = 0;
            for (int t = blockIdx.x; t < ntiles && !abort_flag; t += gridDim.x) {
                int mt, ntl;
                tm.tile(t, mt, ntl);
                if (tm.skip(mt, ntl)) continue;
                for (int kt = 0; kt < nk; kt++, it++) {
                    const int s = it % STAGES;
                    if (!mbar_wait(smem_u32(&empty[s]), ((it / STAGES) & 1) ^ 1, status, &abort_flag)) break;
                    unsigned char* st = smem + s * STAGE_BYTES;
                    const uint32_t fb = smem_u32(&full[s]);
                    mbar_expect_tx(fb, STAGE_BYTES);
                    tma_load_2d(smem_u32(st), &tA_hi, kt * BKE, mt * BM, fb);
                    tma_load_2d(smem_u32(st + A_BYTES), &tA_lo, kt * BKE, mt * BM, fb);
                    tma_load_2d(smem_u32(st + 2 * A_BYTES), &tB_hi, kt * BKE, ntl * BN, fb);
                    tma_load_2d(smem_u32(st + 2 * A_BYTES + B_BYTES), &tB_lo, kt * BKE, ntl * BN, fb);
                    issued_total = it + 1;
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            int it = 0, lt = 0;
            for (int t = blockIdx.x; t < ntiles && !abort_flag; t += gridDim.x) {
                {
                    int mt, ntl;
                    tm.tile(t, mt, ntl);
                    if (tm.skip(mt, ntl)) continue;
                }
                const int b = lt & 1;
                lt++;  // accumulator buffers alternate over the tiles this CTA computes
                if (!mbar_wait(smem_u32(&tempty[b]), (((lt - 1) >> 1) & 1) ^ 1, status, &abort_flag)) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t acc = tmem + (uint32_t)(b * 256);
                bool ok = true;
                for (int kt = 0; kt < nk; kt++, it++) {
                    const int s = it % STAGES;
                    if (!mbar_wait(smem_u32(&full[s]), (it / STAGES) & 1, status, &abort_flag)) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    unsigned char* st = smem + s * STAGE_BYTES;
                    const uint32_t a_hi = smem_u32(st), a_lo = smem_u32(st + A_BYTES);
                    const uint32_t b_hi = smem_u32(st + 2 * A_BYTES), b_lo = smem_u32(st + 2 * A_BYTES + B_BYTES);
#pragma unroll
                    for (int ks = 0; ks < BK / 8; ks++) {
                        const uint32_t off = ks * 32;
                        const uint64_t dah = smem_desc(a_hi + off), dal = smem_desc(a_lo + off);
                        const uint64_t dbh = smem_desc(b_hi + off), dbl = smem_desc(b_lo + off);
                        if (F16) {
                            mma_f16(acc, dah, dbh, (kt > 0 || ks > 0) ? 1u : 0u);
                            mma_f16(acc, dah, dbl, 1u);
                            mma_f16(acc, dal, dbh, 1u);
                        } else {
                            mma_tf32(acc, dah, dbh, (kt > 0 || ks > 0) ? 1u : 0u);
                            mma_tf32(acc, dah, dbl, 1u);
                            mma_tf32(acc, dal, dbh, 1u);
                        }
                    }
                    mma_commit(smem_u32(&empty[s]));
                    consumed_total = it + 1;
                }
                mma_commit(smem_u32(&tfull[b]));
                if (!ok) break;
            }
        }
    } else {
        // epilogue warps 2..5: TMEM lane quarter = warp % 4
        const int q = warp & 3;
        // C of the tile after the current one is prefetched into L2 while the
        // tensor cores work on it, so the read-modify-write below hits L2
        auto prefetch_c = [&](int t) {
            if (t >= ntiles || store) return;
            int mt, ntl;
            tm.tile(t, mt, ntl);
            if (tm.skip(mt, ntl)) return;
            const int i = q * 32 + lane;  // 128 threads: one row (row-major C) or one column (column-major C)
            const int c0 = ntl * (BN / 2);
            if (!c_colmajor) {
                const int row = mt * BM + i;
                if (row >= M || c0 >= Nc) return;
                const char* p = reinterpret_cast<const char*>(&C[(int64_t)row * ldc + c0]);
                const int bytes = min(BN / 2, Nc - c0) * (int)sizeof(float2);
                for (int o = 0; o < bytes; o += 128) asm volatile("prefetch.global.L2 [%0];" ::"l"(p + o));
            } else {
                const int col = c0 + i, r0 = mt * BM;
                if (col >= Nc || r0 >= M) return;
                const char* p = reinterpret_cast<const char*>(&C[(int64_t)col * ldc + r0]);
                const int bytes = min(BM, M - r0) * (int)sizeof(float2);
                for (int o = 0; o < bytes; o += 128) asm volatile("prefetch.global.L2 [%0];" ::"l"(p + o));
            }
        };
        prefetch_c(blockIdx.x);
        int lt = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
            {
                int mt, ntl;
                tm.tile(t, mt, ntl);
                if (tm.skip(mt, ntl)) continue;
            }
            const int b = lt & 1;
            const int ph = (lt >> 1) & 1;
            lt++;
            prefetch_c(t + gridDim.x);
            bool ok = mbar_wait(smem_u32(&tfull[b]), ph, status, &abort_flag);
            ok = __all_sync(0xffffffffu, ok);
            if (!ok) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            int mt, ntl;
            tm.tile(t, mt, ntl);
            const int row = mt * BM + q * 32 + lane;
            const uint32_t base = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * 256);
#pragma unroll 1
            for (int ch = 0; ch < BN / 32; ch++) {
                float v[32];
                tmem_ld32(base + ch * 32, v);
                const int c0 = ntl * (BN / 2) + ch * 16;
                if (row < M && c0 < Nc) {
                    if (F16) {
                        // undo the row and column scales (powers of two: exact)
                        const float ra = sa[row].y;
#pragma unroll
                        for (int j = 0; j < 16; j++) {
                            const float f = c0 + j < Nc ? ra * sb[c0 + j].y : 0.f;
                            v[2 * j] *= f;
                            v[2 * j + 1] *= f;
                        }
                    }
                    if (!c_colmajor) {
                        float2* p = &C[(int64_t)row * ldc + c0];
                        const bool vec = ((reinterpret_cast<uintptr_t>(p) & 15) == 0) && (c0 + 16 <= Nc);
                        if (vec) {
                            // all loads first: the chunk's eight 16-byte reads are in flight together
                            float4* p4 = reinterpret_cast<float4*>(p);
                            float4 c[8];
#pragma unroll
                            for (int j = 0; j < 8; j++) c[j] = store ? make_float4(0.f, 0.f, 0.f, 0.f) : p4[j];
#pragma unroll
                            for (int j = 0; j < 8; j++) {
                                c[j].x -= v[4 * j];
                                c[j].y -= v[4 * j + 1];
                                c[j].z -= v[4 * j + 2];
                                c[j].w -= v[4 * j + 3];
                                p4[j] = c[j];
                            }
                        } else {
#pragma unroll
                            for (int j = 0; j < 16; j++)
                                if (c0 + j < Nc) {
                                    float2 c = store ? make_float2(0.f, 0.f) : p[j];
                                    c.x -= v[2 * j];
                                    c.y -= v[2 * j + 1];
                                    p[j] = c;
                                }
                        }
                    } else {
                        // column-major C: each j is one coalesced 256-byte row segment of the warp;
                        // issue the 16 reads before any write
                        const int nj = min(16, Nc - c0);
                        float2 c[16];
#pragma unroll
                        for (int j = 0; j < 16; j++)
                            if (j < nj) c[j] = store ? make_float2(0.f, 0.f) : C[(int64_t)(c0 + j) * ldc + row];
#pragma unroll
                        for (int j = 0; j < 16; j++)
                            if (j < nj) {
                                c[j].x -= v[2 * j];
                                c[j].y -= v[2 * j + 1];
                                C[(int64_t)(c0 + j) * ldc + row] = c[j];
                            }
                    }
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&tempty[b]));
        }
    }
    __syncwarp();
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    // teardown: on an aborted run, let the copies already issued land
    if (threadIdx.x == 0 && abort_flag) {
        for (int it = consumed_total; it < issued_total; it++) {
            long long t0 = clock64();
            while (!mbar_try(smem_u32(&full[it % STAGES]), (it / STAGES) & 1) && clock64() - t0 < WAIT_CYCLES) {
            }
        }
    }
    __syncthreads();
    if (warp == 1) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS2));
    }
}

// ------------------------------------------------------- CTA pairs (cta_group::2)
// FP16-part products on clusters of two CTAs (one TPC): a 256-row x 256-column
// tile, each CTA loading its 128 rows of A (hi, lo) and 128 of the tile's 256
// B' rows (hi, lo), the even CTA issuing tcgen05.mma.cta_group::2 (M = 256,
// N = 256), which reads both CTAs' shared memory and accumulates each CTA's
// 128 rows in its own TMEM.  A stage is 64 KB per CTA (96 KB for the one-CTA
// tile, whose B is not shared), so three stages fit: per SM, 64 KB of operands
// per 384 MMA cycles against 96 KB.  Barriers: full[s] lives on the even CTA
// and expects both CTAs' bytes (one arrival, its producer's, plus the
// transactions of both CTAs' .cta_group::2 loads); empty[s] and tfull[b]
// receive the MMA commits multicast to the pair; tempty[b] on the even CTA
// counts the epilogue warps of both.  No load is multicast.  Eight epilogue
// warps per CTA: two per TMEM lane quarter, each draining half of the
// accumulator's columns, so a tile's epilogue takes half as long as with four.
constexpr int P_ROWS = 128;                               // A rows per CTA
constexpr int P_BROWS = 128;                              // B' rows per CTA
constexpr int P_STAGES = 3;
constexpr int P_A_BYTES = P_ROWS * 128;                   // 16 KB per part
constexpr int P_B_BYTES = P_BROWS * 128;                  // 16 KB per part
constexpr int P_STAGE_BYTES = 2 * P_A_BYTES + 2 * P_B_BYTES;  // 64 KB
constexpr int P_EPI_WARPS = 8;                            // epilogue warps per CTA (2 per lane quarter)
constexpr int P_THREADS = 64 + 32 * P_EPI_WARPS;           // producer, MMA issuer, epilogue
constexpr int P_SMEM_BYTES = P_STAGES * P_STAGE_BYTES + 1024 + 256;
constexpr uint32_t P_IDESC_F16 = (1u << 4) | (0u << 7) | (0u << 10) | ((uint32_t)(256 >> 3) << 17) |
                                 ((uint32_t)(256 >> 4) << 24);

__device__ __forceinline__ uint32_t cl_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ uint32_t cl_idx() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(r));
    return r;
}
__device__ __forceinline__ uint32_t cl_count() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%nclusterid.x;" : "=r"(r));
    return r;
}
__device__ __forceinline__ uint32_t cl_map(uint32_t addr, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
    return r;
}
__device__ __forceinline__ void cl_sync() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// TMA load into this CTA's shared memory, its bytes counted on the even CTA's barrier
__device__ __forceinline__ void tma_load_pair(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, "
        "%3}], [%4];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}
__device__ __forceinline__ void mma_f16_pair(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t accumulate) {
    uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8, %9, %10, %11, %12}, p;\n\t}" ::"r"(
            tmem_d),
        "l"(a), "l"(b), "r"(P_IDESC_F16), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z), "r"(z), "r"(z), "r"(z),
        "r"(z));
}
// arrive on the barrier at this shared offset in both CTAs of the pair
__device__ __forceinline__ void mma_commit_pair(uint32_t bar) {
    asm volatile(
        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(bar),
        "h"((uint16_t)3)
        : "memory");
}
__device__ __forceinline__ void mbar_arrive_remote(uint32_t bar_cluster) {
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(bar_cluster) : "memory");
}

// Tiles of 256 rows x 128 complex columns in groups of gm row tiles, column
// by column.  Lower (square row-major C): a group's columns stop at its last
// row's diagonal, and tiles wholly above the diagonal (nt >= 2 mt + 2) are
// skipped by every role alike.
struct PairTiles {
    int num_m, num_n, gm, lower;
    __device__ __forceinline__ int gwidth(int g) const {
        const int first = g * gm, gs = min(gm, num_m - first);
        return lower ? min(num_n, 2 * (first + gs)) : num_n;
    }
    __device__ __forceinline__ int count() const {
        int c = 0;
        for (int g = 0; g * gm < num_m; g++) c += min(gm, num_m - g * gm) * gwidth(g);
        return c;
    }
    __device__ __forceinline__ bool tile(int t, int& mt, int& nt) const {
        int g = 0;
        for (;; g++) {
            const int c = min(gm, num_m - g * gm) * gwidth(g);
            if (t < c) break;
            t -= c;
        }
        const int first = g * gm, gs = min(gm, num_m - first);
        mt = first + t % gs;
        nt = t / gs;
        return !(lower && nt >= 2 * mt + 2);
    }
};

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(P_THREADS, 1)
gemm_pair_kernel(const __grid_constant__ CUtensorMap tA_hi, const __grid_constant__ CUtensorMap tA_lo,
                 const __grid_constant__ CUtensorMap tB_hi, const __grid_constant__ CUtensorMap tB_lo,
                 float2* __restrict__ C, int64_t ldc, int c_colmajor, int M, int Nc, int K2, int lower, int store,
                 int group_m, int* status, const float2* __restrict__ sa, const float2* __restrict__ sb) {
    constexpr int BKE = 2 * BK;  // halves of K per stage (one 128-byte row)
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t* bars = (uint64_t*)(smem + P_STAGES * P_STAGE_BYTES);
    uint64_t* full = bars;                    // [P_STAGES], used in the even CTA
    uint64_t* empty = bars + P_STAGES;        // [P_STAGES]
    uint64_t* tfull = bars + 2 * P_STAGES;    // [2]
    uint64_t* tempty = bars + 2 * P_STAGES + 2;  // [2], used in the even CTA
    uint32_t* tmem_slot = (uint32_t*)(bars + 2 * P_STAGES + 4);
    __shared__ volatile int abort_flag;
    __shared__ int issued_total, consumed_total;

    const uint32_t rank = cl_rank();
    const bool even = rank == 0;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nk = (K2 + BKE - 1) / BKE;
    PairTiles tm;
    tm.num_m = (M + 2 * P_ROWS - 1) / (2 * P_ROWS);
    tm.num_n = (2 * Nc + 2 * P_BROWS - 1) / (2 * P_BROWS);
    tm.gm = group_m > 0 ? group_m : 8;
    tm.lower = lower;
    const int ntiles = tm.count();
    const int cid = (int)cl_idx(), ncl = (int)cl_count();

    if (threadIdx.x == 0) {
        abort_flag = 0;
        issued_total = consumed_total = 0;
        for (int s = 0; s < P_STAGES; s++) {
            mbar_init(smem_u32(&full[s]), 1);
            mbar_init(smem_u32(&empty[s]), 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(smem_u32(&tfull[b]), 1);
            mbar_init(smem_u32(&tempty[b]), 2 * P_EPI_WARPS);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TMEM_COLS2));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    cl_sync();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            int it = 0;
            for (int t = cid; t < ntiles && !abort_flag; t += ncl) {
                int mt, nt;
                if (!tm.tile(t, mt, nt)) continue;
                const int ya = mt * 2 * P_ROWS + (int)rank * P_ROWS;
                const int yb = nt * 2 * P_BROWS + (int)rank * P_BROWS;
                for (int kt = 0; kt < nk; kt++, it++) {
                    const int s = it % P_STAGES;
                    if (!mbar_wait(smem_u32(&empty[s]), ((it / P_STAGES) & 1) ^ 1, status, &abort_flag)) break;
                    unsigned char* st = smem + s * P_STAGE_BYTES;
                    const uint32_t fb = cl_map(smem_u32(&full[s]), 0);
                    if (even) mbar_expect_tx(smem_u32(&full[s]), 2 * P_STAGE_BYTES);
                    tma_load_pair(smem_u32(st), &tA_hi, kt * BKE, ya, fb);
                    tma_load_pair(smem_u32(st + P_A_BYTES), &tA_lo, kt * BKE, ya, fb);
                    tma_load_pair(smem_u32(st + 2 * P_A_BYTES), &tB_hi, kt * BKE, yb, fb);
                    tma_load_pair(smem_u32(st + 2 * P_A_BYTES + P_B_BYTES), &tB_lo, kt * BKE, yb, fb);
                    issued_total = it + 1;
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0 && even) {
            int it = 0, lt = 0;
            for (int t = cid; t < ntiles && !abort_flag; t += ncl) {
                int mt, nt;
                if (!tm.tile(t, mt, nt)) continue;
                const int b = lt & 1;
                lt++;
                if (!mbar_wait(smem_u32(&tempty[b]), (((lt - 1) >> 1) & 1) ^ 1, status, &abort_flag)) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t acc = tmem + (uint32_t)(b * 256);
                bool ok = true;
                for (int kt = 0; kt < nk; kt++, it++) {
                    const int s = it % P_STAGES;
                    if (!mbar_wait(smem_u32(&full[s]), (it / P_STAGES) & 1, status, &abort_flag)) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    unsigned char* st = smem + s * P_STAGE_BYTES;
                    const uint32_t a_hi = smem_u32(st), a_lo = smem_u32(st + P_A_BYTES);
                    const uint32_t b_hi = smem_u32(st + 2 * P_A_BYTES), b_lo = smem_u32(st + 2 * P_A_BYTES + P_B_BYTES);
#pragma unroll
                    for (int ks = 0; ks < BK / 8; ks++) {
                        const uint32_t off = ks * 32;
                        const uint64_t dah = smem_desc(a_hi + off), dal = smem_desc(a_lo + off);
                        const uint64_t dbh = smem_desc(b_hi + off), dbl = smem_desc(b_lo + off);
                        mma_f16_pair(acc, dah, dbh, (kt > 0 || ks > 0) ? 1u : 0u);
                        mma_f16_pair(acc, dah, dbl, 1u);
                        mma_f16_pair(acc, dal, dbh, 1u);
                    }
                    mma_commit_pair(smem_u32(&empty[s]));
                    consumed_total = it + 1;
                }
                mma_commit_pair(smem_u32(&tfull[b]));
                if (!ok) break;
            }
        }
    } else {
        // epilogue warps 2..9 of both CTAs: TMEM lane quarter = warp % 4, and
        // half of the 256 accumulator columns each
        // chunks [ch0, ch1) of the 8 32-column chunks for this warp
        const int q = warp & 3, part = (warp - 2) >> 2, nparts = P_EPI_WARPS / 4;
        const int ch0 = part * 8 / nparts, ch1 = (part + 1) * 8 / nparts;
        const uint32_t te0 = cl_map(smem_u32(&tempty[0]), 0), te1 = cl_map(smem_u32(&tempty[1]), 0);
        int lt = 0;
        for (int t = cid; t < ntiles; t += ncl) {
            int mt, nt;
            if (!tm.tile(t, mt, nt)) continue;
            const int b = lt & 1;
            const int ph = (lt >> 1) & 1;
            lt++;
            bool ok = mbar_wait(smem_u32(&tfull[b]), ph, status, &abort_flag);
            ok = __all_sync(0xffffffffu, ok);
            if (!ok) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            // lower: this CTA's 128 rows wholly above the diagonal are not written
            const bool write = !(lower && nt >= 2 * mt + (int)rank + 1);
            const int row = mt * 2 * P_ROWS + (int)rank * P_ROWS + q * 32 + lane;
            const uint32_t base = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * 256);
#pragma unroll 1
            for (int ch = ch0; ch < ch1 && write; ch++) {
                float v[32];
                tmem_ld32(base + ch * 32, v);
                const int c0 = nt * P_BROWS + ch * 16;
                if (row < M && c0 < Nc) {
                    const float ra = sa[row].y;
#pragma unroll
                    for (int j = 0; j < 16; j++) {
                        const float f = c0 + j < Nc ? ra * sb[c0 + j].y : 0.f;
                        v[2 * j] *= f;
                        v[2 * j + 1] *= f;
                    }
                    if (!c_colmajor) {
                        float2* p = &C[(int64_t)row * ldc + c0];
                        const bool vec = ((reinterpret_cast<uintptr_t>(p) & 15) == 0) && (c0 + 16 <= Nc);
                        if (vec) {
                            float4* p4 = reinterpret_cast<float4*>(p);
                            float4 c[8];
#pragma unroll
                            for (int j = 0; j < 8; j++) c[j] = store ? make_float4(0.f, 0.f, 0.f, 0.f) : p4[j];
#pragma unroll
                            for (int j = 0; j < 8; j++) {
                                c[j].x -= v[4 * j];
                                c[j].y -= v[4 * j + 1];
                                c[j].z -= v[4 * j + 2];
                                c[j].w -= v[4 * j + 3];
                                p4[j] = c[j];
                            }
                        } else {
#pragma unroll
                            for (int j = 0; j < 16; j++)
                                if (c0 + j < Nc) {
                                    float2 c = store ? make_float2(0.f, 0.f) : p[j];
                                    c.x -= v[2 * j];
                                    c.y -= v[2 * j + 1];
                                    p[j] = c;
                                }
                        }
                    } else {
                        const int nj = min(16, Nc - c0);
                        float2 c[16];
#pragma unroll
                        for (int j = 0; j < 16; j++)
                            if (j < nj) c[j] = store ? make_float2(0.f, 0.f) : C[(int64_t)(c0 + j) * ldc + row];
#pragma unroll
                        for (int j = 0; j < 16; j++)
                            if (j < nj) {
                                c[j].x -= v[2 * j];
                                c[j].y -= v[2 * j + 1];
                                C[(int64_t)(c0 + j) * ldc + row] = c[j];
                            }
                    }
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive_remote(b ? te1 : te0);
        }
    }
    __syncwarp();
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    // an aborted run: let the copies counted on the even CTA's barriers land
    if (threadIdx.x == 0 && abort_flag && even) {
        for (int it = consumed_total; it < issued_total; it++) {
            long long t0 = clock64();
            while (!mbar_try(smem_u32(&full[it % P_STAGES]), (it / P_STAGES) & 1) && clock64() - t0 < WAIT_CYCLES) {
            }
        }
    }
    cl_sync();
    if (warp == 1) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS2));
    }
    cl_sync();
}

// ---------------------------------------------------------------- packing
// A (complex, K contiguous): hi/lo[i*ld + 2k + {0,1}] = split(Re/Im a_ik), zero padded
__global__ void pack_a_kernel(const float2* __restrict__ A, int64_t lda, int M, int K, float* __restrict__ hi,
                              float* __restrict__ lo, int ld) {
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t tot = (int64_t)M * (ld / 2);
    if (t >= tot) return;
    int i = (int)(t / (ld / 2)), k = (int)(t % (ld / 2));
    float2 a = k < K ? A[(int64_t)i * lda + k] : make_float2(0.f, 0.f);
    float h0 = to_tf32(a.x), h1 = to_tf32(a.y);
    float l0 = to_tf32(a.x - h0), l1 = to_tf32(a.y - h1);
    reinterpret_cast<float2*>(hi + (int64_t)i * ld)[k] = make_float2(h0, h1);
    reinterpret_cast<float2*>(lo + (int64_t)i * ld)[k] = make_float2(l0, l1);
}

// A given as its transpose (At: K x M row-major, A[i][k] = At[k*lda + i]),
// transposed through shared memory into the K-major hi / lo planes.
__global__ void pack_a_trans_kernel(const float2* __restrict__ At, int64_t lda, int M, int K, float* __restrict__ hi,
                                    float* __restrict__ lo, int ld) {
    __shared__ float2 tile[32][33];
    const int i0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 256 threads: 8 rows per pass
    for (int r = ty; r < 32; r += 8) {
        int k = k0 + r, i = i0 + tx;
        tile[r][tx] = (k < K && i < M) ? At[(int64_t)k * lda + i] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        int i = i0 + r, k = k0 + tx;
        if (i >= M || k >= ld / 2) continue;
        float2 a = tile[tx][r];
        float h0 = to_tf32(a.x), h1 = to_tf32(a.y);
        float l0 = to_tf32(a.x - h0), l1 = to_tf32(a.y - h1);
        reinterpret_cast<float2*>(hi + (int64_t)i * ld)[k] = make_float2(h0, h1);
        reinterpret_cast<float2*>(lo + (int64_t)i * ld)[k] = make_float2(l0, l1);
    }
}

// B given column-major (B[j*ldb + k], K contiguous): rows 2j, 2j+1 of B'.
// With `dsc`, B[k][j] is multiplied by the complex factor dsc[k * dstride]
// first (the D of an L D L^T update, read from the factor's diagonal).
__global__ void pack_b_col_kernel(const float2* __restrict__ B, int64_t ldb, int N, int K, float* __restrict__ hi,
                                  float* __restrict__ lo, int ld, const float2* __restrict__ dsc, int64_t dstride) {
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t tot = (int64_t)N * (ld / 2);
    if (t >= tot) return;
    int j = (int)(t / (ld / 2)), k = (int)(t % (ld / 2));
    float2 b = k < K ? B[(int64_t)j * ldb + k] : make_float2(0.f, 0.f);
    if (dsc && k < K) {
        const float2 d = dsc[(int64_t)k * dstride];
        b = make_float2(b.x * d.x - b.y * d.y, b.x * d.y + b.y * d.x);
    }
    float hr = to_tf32(b.x), hi_ = to_tf32(b.y);
    float lr = to_tf32(b.x - hr), li = to_tf32(b.y - hi_);
    float2* r0h = reinterpret_cast<float2*>(hi + (int64_t)(2 * j) * ld);
    float2* r1h = reinterpret_cast<float2*>(hi + (int64_t)(2 * j + 1) * ld);
    float2* r0l = reinterpret_cast<float2*>(lo + (int64_t)(2 * j) * ld);
    float2* r1l = reinterpret_cast<float2*>(lo + (int64_t)(2 * j + 1) * ld);
    r0h[k] = make_float2(hr, -hi_);
    r1h[k] = make_float2(hi_, hr);
    r0l[k] = make_float2(lr, -li);
    r1l[k] = make_float2(li, lr);
}

// B given row-major (B[k*ldb + j], N contiguous): transposed through shared memory.
__global__ void pack_b_row_kernel(const float2* __restrict__ B, int64_t ldb, int N, int K, float* __restrict__ hi,
                                  float* __restrict__ lo, int ld) {
    __shared__ float2 tile[32][33];
    const int j0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 256 threads: 8 rows per pass
    for (int r = ty; r < 32; r += 8) {
        int k = k0 + r, j = j0 + tx;
        tile[r][tx] = (k < K && j < N) ? B[(int64_t)k * ldb + j] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        int j = j0 + r, k = k0 + tx;
        if (j >= N || k >= ld / 2) continue;
        float2 b = tile[tx][r];
        float hr = to_tf32(b.x), hi_ = to_tf32(b.y);
        float lr = to_tf32(b.x - hr), li = to_tf32(b.y - hi_);
        reinterpret_cast<float2*>(hi + (int64_t)(2 * j) * ld)[k] = make_float2(hr, -hi_);
        reinterpret_cast<float2*>(hi + (int64_t)(2 * j + 1) * ld)[k] = make_float2(hi_, hr);
        reinterpret_cast<float2*>(lo + (int64_t)(2 * j) * ld)[k] = make_float2(lr, -li);
        reinterpret_cast<float2*>(lo + (int64_t)(2 * j + 1) * ld)[k] = make_float2(li, lr);
    }
}

// ---------------------------------------------------------------- FP16 split
// Scale of one operand row (A') or complex column (B): the power of two s
// with s * max(|Re|, |Im|) in [2^14, 2^15), stored with its inverse as
// sc[t] = (s, 1/s).  Element k of item t is X[t * si + k * sk], times
// dsc[k * dstride] when dsc is given (the D of an L D L^T update, applied as
// the pack kernel applies it).  per_warp: one warp per item, lanes over k
// (k contiguous); else 32 items per block of 256 threads (items contiguous
// across the lanes of a warp), the 8 warps over interleaved k, reduced in
// shared memory.
__global__ void f16_scale_kernel(const float2* __restrict__ X, int64_t si, int64_t sk, int n, int K,
                                 const float2* __restrict__ dsc, int64_t dstride, int per_warp,
                                 float2* __restrict__ sc) {
    float m = 0.f;
    int t;
    int k0 = 0, kstep = 1;
    if (per_warp) {
        t = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
        k0 = threadIdx.x & 31;
        kstep = 32;
    } else {
        t = (int)blockIdx.x * 32 + (int)(threadIdx.x & 31);
        k0 = (int)(threadIdx.x >> 5);
        kstep = (int)(blockDim.x >> 5);
    }
    if (t < n) {
        for (int k = k0; k < K; k += kstep) {
            float2 x = X[(int64_t)t * si + (int64_t)k * sk];
            if (dsc) {
                const float2 d = dsc[(int64_t)k * dstride];
                x = make_float2(x.x * d.x - x.y * d.y, x.x * d.y + x.y * d.x);
            }
            m = fmaxf(m, fmaxf(fabsf(x.x), fabsf(x.y)));
        }
    }
    if (per_warp) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
        if ((threadIdx.x & 31) != 0) return;
    } else {
        __shared__ float part[32][33];
        part[threadIdx.x >> 5][threadIdx.x & 31] = m;
        __syncthreads();
        if (threadIdx.x >= 32) return;
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) m = fmaxf(m, part[w][threadIdx.x]);
    }
    if (t >= n) return;
    float sv = 1.f, inv = 1.f;
    if (m > 0.f && m <= 3.0e38f) {
        int e;
        frexpf(m, &e);  // m = f 2^e, f in [0.5, 1)
        e = max(e, -100);
        sv = ldexpf(1.f, 15 - e);
        inv = ldexpf(1.f, e - 15);
    }
    sc[t] = make_float2(sv, inv);
}

__device__ __forceinline__ void split_h(float x, __half& h, __half& l) {
    h = __float2half_rn(x);
    l = __float2half_rn(x - __half2float(h));
}

// The FP16 counterparts of the four pack kernels above: same layouts, each
// value multiplied by its row's (A) or column's (B) scale first.
__global__ void pack_a_h_kernel(const float2* __restrict__ A, int64_t lda, int M, int K, __half* __restrict__ hi,
                                __half* __restrict__ lo, int ld, const float2* __restrict__ sc) {
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t tot = (int64_t)M * (ld / 2);
    if (t >= tot) return;
    int i = (int)(t / (ld / 2)), k = (int)(t % (ld / 2));
    float2 a = k < K ? A[(int64_t)i * lda + k] : make_float2(0.f, 0.f);
    const float s = sc[i].x;
    __half h0, h1, l0, l1;
    split_h(a.x * s, h0, l0);
    split_h(a.y * s, h1, l1);
    reinterpret_cast<__half2*>(hi + (int64_t)i * ld)[k] = __halves2half2(h0, h1);
    reinterpret_cast<__half2*>(lo + (int64_t)i * ld)[k] = __halves2half2(l0, l1);
}

__global__ void pack_a_trans_h_kernel(const float2* __restrict__ At, int64_t lda, int M, int K,
                                      __half* __restrict__ hi, __half* __restrict__ lo, int ld,
                                      const float2* __restrict__ sc) {
    __shared__ float2 tile[32][33];
    const int i0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int r = ty; r < 32; r += 8) {
        int k = k0 + r, i = i0 + tx;
        tile[r][tx] = (k < K && i < M) ? At[(int64_t)k * lda + i] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        int i = i0 + r, k = k0 + tx;
        if (i >= M || k >= ld / 2) continue;
        float2 a = tile[tx][r];
        const float s = sc[i].x;
        __half h0, h1, l0, l1;
        split_h(a.x * s, h0, l0);
        split_h(a.y * s, h1, l1);
        reinterpret_cast<__half2*>(hi + (int64_t)i * ld)[k] = __halves2half2(h0, h1);
        reinterpret_cast<__half2*>(lo + (int64_t)i * ld)[k] = __halves2half2(l0, l1);
    }
}

__global__ void pack_b_col_h_kernel(const float2* __restrict__ B, int64_t ldb, int N, int K, __half* __restrict__ hi,
                                    __half* __restrict__ lo, int ld, const float2* __restrict__ dsc,
                                    int64_t dstride, const float2* __restrict__ sc) {
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t tot = (int64_t)N * (ld / 2);
    if (t >= tot) return;
    int j = (int)(t / (ld / 2)), k = (int)(t % (ld / 2));
    float2 b = k < K ? B[(int64_t)j * ldb + k] : make_float2(0.f, 0.f);
    if (dsc && k < K) {
        const float2 d = dsc[(int64_t)k * dstride];
        b = make_float2(b.x * d.x - b.y * d.y, b.x * d.y + b.y * d.x);
    }
    const float s = sc[j].x;
    __half hr, hm, lr, lm;
    split_h(b.x * s, hr, lr);
    split_h(b.y * s, hm, lm);
    reinterpret_cast<__half2*>(hi + (int64_t)(2 * j) * ld)[k] = __halves2half2(hr, __hneg(hm));
    reinterpret_cast<__half2*>(hi + (int64_t)(2 * j + 1) * ld)[k] = __halves2half2(hm, hr);
    reinterpret_cast<__half2*>(lo + (int64_t)(2 * j) * ld)[k] = __halves2half2(lr, __hneg(lm));
    reinterpret_cast<__half2*>(lo + (int64_t)(2 * j + 1) * ld)[k] = __halves2half2(lm, lr);
}

__global__ void pack_b_row_h_kernel(const float2* __restrict__ B, int64_t ldb, int N, int K, __half* __restrict__ hi,
                                    __half* __restrict__ lo, int ld, const float2* __restrict__ sc) {
    __shared__ float2 tile[32][33];
    const int j0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int r = ty; r < 32; r += 8) {
        int k = k0 + r, j = j0 + tx;
        tile[r][tx] = (k < K && j < N) ? B[(int64_t)k * ldb + j] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        int j = j0 + r, k = k0 + tx;
        if (j >= N || k >= ld / 2) continue;
        float2 b = tile[tx][r];
        const float s = sc[j].x;
        __half hr, hm, lr, lm;
        split_h(b.x * s, hr, lr);
        split_h(b.y * s, hm, lm);
        reinterpret_cast<__half2*>(hi + (int64_t)(2 * j) * ld)[k] = __halves2half2(hr, __hneg(hm));
        reinterpret_cast<__half2*>(hi + (int64_t)(2 * j + 1) * ld)[k] = __halves2half2(hm, hr);
        reinterpret_cast<__half2*>(lo + (int64_t)(2 * j) * ld)[k] = __halves2half2(lr, __hneg(lm));
        reinterpret_cast<__half2*>(lo + (int64_t)(2 * j + 1) * ld)[k] = __halves2half2(lm, lr);
    }
}

}  // namespace tc

// ---------------------------------------------------------------- host side
static PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

static int tc_encode_init(bem_ctx* ctx) {
    if (g_encode) return BEM_OK;
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    BEM_TRY_CUDA(ctx, cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
    if (q != cudaDriverEntryPointSuccess || !fn)
        return fail(ctx, BEM_ERR_CUDA, "cuTensorMapEncodeTiled entry point unavailable");
    g_encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    return BEM_OK;
}

// One operand plane: rows x ld elements (FP32, or FP16 when f16), rows of
// 128 bytes per box (32 floats or 64 halves), 128-byte swizzle.
static int make_map(bem_ctx* ctx, CUtensorMap* map, void* base, int rows, int ld, int box_rows, bool f16 = false) {
    const int esz = f16 ? 2 : 4;
    cuuint64_t dims[2] = {(cuuint64_t)ld, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)ld * esz};
    cuuint32_t box[2] = {(cuuint32_t)(128 / esz), (cuuint32_t)box_rows};
    cuuint32_t es[2] = {1, 1};
    CUresult r = g_encode(map, f16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, base,
                           dims, strides, box, es,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(ctx, BEM_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return BEM_OK;
}

// C -= A * B on the tensor cores.  b_rowmajor: B[k*ldb + j] (U12 block),
// else B[j*ldb + k].  c_colmajor: C[j*ldc + i], else C[i*ldc + j].
int tc_gemm_ex(bem_ctx* ctx, int M, int N, int K, const float2* A, int64_t lda, const float2* B, int64_t ldb,
               float2* C, int64_t ldc, const TcOpts& o) {
    const bool b_rowmajor = o.b_rowmajor, c_colmajor = o.c_colmajor;
    const int prof_cls = o.prof_cls;
    if (M <= 0 || N <= 0 || K <= 0) return BEM_OK;
    if (o.lower && (M != N || c_colmajor)) return fail(ctx, BEM_ERR_INVALID, "tc gemm: lower needs square row-major C");
    if (o.bscale && b_rowmajor) return fail(ctx, BEM_ERR_INVALID, "tc gemm: B scaling needs column-major B");
    BEM_TRY(tc_encode_init(ctx));
    // FP16 parts need the persistent kernel; the one-CTA-per-tile kernel keeps TF32
    const bool f16 = ctx->tc_split == 1 && ctx->tc_persistent;
    const size_t esz = f16 ? 2 : 4;
    const int bke = f16 ? 2 * tc::BK : tc::BK;  // elements per 128-byte row
    // K-major operand rows padded to a multiple of 128 bytes
    const int ld = ((2 * K + bke - 1) / bke) * bke;
    size_t a_elems = (size_t)M * ld, b_elems = (size_t)2 * N * ld;
    const size_t planes = 2 * (a_elems + b_elems) * esz;
    const size_t sc_off = (planes + 255) & ~(size_t)255;
    size_t need = (f16 ? sc_off + (size_t)(M + N) * sizeof(float2) : planes) + 1024;
    if (need > ctx->tc_bytes) {
        if (ctx->tc_buf) {
            BEM_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            cudaFree(ctx->tc_buf);
        }
        ctx->tc_buf = nullptr;
        ctx->tc_bytes = 0;
        BEM_TRY_CUDA(ctx, cudaMalloc(&ctx->tc_buf, need));
        ctx->tc_bytes = need;
    }
    char* base = reinterpret_cast<char*>(ctx->tc_buf);
    void* a_hi = base;
    void* a_lo = base + a_elems * esz;
    void* b_hi = base + 2 * a_elems * esz;
    void* b_lo = base + (2 * a_elems + b_elems) * esz;
    float2* sc_a = f16 ? reinterpret_cast<float2*>(base + sc_off) : nullptr;
    float2* sc_b = f16 ? sc_a + M : nullptr;
    cudaEvent_t ev = prof_cls >= 0 ? ctx->prof_begin(prof_cls) : nullptr;
    if (f16) {
        // scales: rows of A (k contiguous unless A comes transposed), complex columns of B
        if (o.a_trans)
            tc::f16_scale_kernel<<<(M + 31) / 32, 256, 0, ctx->stream>>>(A, 1, lda, M, K, nullptr, 0, 0, sc_a);
        else
            tc::f16_scale_kernel<<<(unsigned)(((int64_t)M * 32 + 255) / 256), 256, 0, ctx->stream>>>(
                A, lda, 1, M, K, nullptr, 0, 1, sc_a);
        BEM_LAUNCHED(ctx);
        if (b_rowmajor)
            tc::f16_scale_kernel<<<(N + 31) / 32, 256, 0, ctx->stream>>>(B, 1, ldb, N, K, nullptr, 0, 0, sc_b);
        else
            tc::f16_scale_kernel<<<(unsigned)(((int64_t)N * 32 + 255) / 256), 256, 0, ctx->stream>>>(
                B, ldb, 1, N, K, o.bscale, o.bscale_stride, 1, sc_b);
        BEM_LAUNCHED(ctx);
        __half *ah = (__half*)a_hi, *al = (__half*)a_lo, *bh = (__half*)b_hi, *bl = (__half*)b_lo;
        if (o.a_trans) {
            dim3 g((M + 31) / 32, (ld / 2 + 31) / 32);
            tc::pack_a_trans_h_kernel<<<g, 256, 0, ctx->stream>>>(A, lda, M, K, ah, al, ld, sc_a);
        } else {
            int64_t tot = (int64_t)M * (ld / 2);
            tc::pack_a_h_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, ctx->stream>>>(A, lda, M, K, ah, al, ld,
                                                                                       sc_a);
        }
        BEM_LAUNCHED(ctx);
        if (b_rowmajor) {
            dim3 g((N + 31) / 32, (ld / 2 + 31) / 32);
            tc::pack_b_row_h_kernel<<<g, 256, 0, ctx->stream>>>(B, ldb, N, K, bh, bl, ld, sc_b);
        } else {
            int64_t tot = (int64_t)N * (ld / 2);
            tc::pack_b_col_h_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, ctx->stream>>>(
                B, ldb, N, K, bh, bl, ld, o.bscale, o.bscale_stride, sc_b);
        }
        BEM_LAUNCHED(ctx);
    } else {
        float *ah = (float*)a_hi, *al = (float*)a_lo, *bh = (float*)b_hi, *bl = (float*)b_lo;
        if (o.a_trans) {
            dim3 g((M + 31) / 32, (ld / 2 + 31) / 32);
            tc::pack_a_trans_kernel<<<g, 256, 0, ctx->stream>>>(A, lda, M, K, ah, al, ld);
            BEM_LAUNCHED(ctx);
        } else {
            int64_t tot = (int64_t)M * (ld / 2);
            tc::pack_a_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, ctx->stream>>>(A, lda, M, K, ah, al, ld);
            BEM_LAUNCHED(ctx);
        }
        if (b_rowmajor) {
            dim3 g((N + 31) / 32, (ld / 2 + 31) / 32);
            tc::pack_b_row_kernel<<<g, 256, 0, ctx->stream>>>(B, ldb, N, K, bh, bl, ld);
        } else {
            int64_t tot = (int64_t)N * (ld / 2);
            tc::pack_b_col_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, ctx->stream>>>(B, ldb, N, K, bh, bl, ld,
                                                                                         o.bscale, o.bscale_stride);
        }
        BEM_LAUNCHED(ctx);
    }
    CUtensorMap mah, mal, mbh, mbl;
    BEM_TRY(make_map(ctx, &mah, a_hi, M, ld, tc::BM, f16));
    BEM_TRY(make_map(ctx, &mal, a_lo, M, ld, tc::BM, f16));
    BEM_TRY(make_map(ctx, &mbh, b_hi, 2 * N, ld, tc::BN, f16));
    BEM_TRY(make_map(ctx, &mbl, b_lo, 2 * N, ld, tc::BN, f16));
    if (!ctx->tc_attr) {
        BEM_TRY_CUDA(ctx, cudaFuncSetAttribute(tc::gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               tc::SMEM_BYTES));
        BEM_TRY_CUDA(ctx, cudaFuncSetAttribute(tc::gemm_persistent_kernel<false>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, tc::SMEM_BYTES));
        BEM_TRY_CUDA(ctx, cudaFuncSetAttribute(tc::gemm_persistent_kernel<true>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, tc::SMEM_BYTES));
        ctx->tc_attr = true;
    }
    if (f16 && ctx->tc_pair) {
        // 128-row B' boxes: each CTA of a pair loads half of the tile's 256 B' rows
        CUtensorMap pbh, pbl;
        BEM_TRY(make_map(ctx, &pbh, b_hi, 2 * N, ld, tc::P_BROWS, true));
        BEM_TRY(make_map(ctx, &pbl, b_lo, 2 * N, ld, tc::P_BROWS, true));
        if (!ctx->tc_pair_attr) {
            BEM_TRY_CUDA(ctx, cudaFuncSetAttribute(tc::gemm_pair_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   tc::P_SMEM_BYTES));
            ctx->tc_pair_attr = true;
        }
        const int nm = (M + 2 * tc::P_ROWS - 1) / (2 * tc::P_ROWS), nn = (2 * N + 255) / 256;
        const int ntiles = o.lower ? nm * std::min(nn, 2 * nm) : nm * nn;  // an upper bound for the lower raster
        const int grid = 2 * std::max(1, std::min(ntiles, ctx->sm_count / 2));
        tc::gemm_pair_kernel<<<grid, tc::P_THREADS, tc::P_SMEM_BYTES, ctx->stream>>>(
            mah, mal, pbh, pbl, C, ldc, c_colmajor ? 1 : 0, M, N, ld, o.lower ? 1 : 0, o.store ? 1 : 0,
            std::max(1, ctx->tc_group_m / 2), ctx->d_status, sc_a, sc_b);
    } else if (ctx->tc_persistent) {
        const int nm = (M + tc::BM - 1) / tc::BM;
        const int ntiles = o.lower ? nm * (nm + 1) / 2 : nm * ((2 * N + tc::BN - 1) / tc::BN);
        const int grid = std::min(ntiles, ctx->sm_count);
        auto kern = f16 ? tc::gemm_persistent_kernel<true> : tc::gemm_persistent_kernel<false>;
        kern<<<grid, 192, tc::SMEM_BYTES, ctx->stream>>>(mah, mal, mbh, mbl, C, ldc, c_colmajor ? 1 : 0, M, N, ld,
                                                         o.lower ? 1 : 0, o.store ? 1 : 0, ctx->tc_group_m,
                                                         ctx->d_status, sc_a, sc_b);
    } else {
        dim3 grid((2 * N + tc::BN - 1) / tc::BN, (M + tc::BM - 1) / tc::BM);
        if (grid.y > 65535) return fail(ctx, BEM_ERR_INVALID, "tc gemm: M too large");
        if (o.lower || o.store) return fail(ctx, BEM_ERR_INVALID, "tc gemm: lower / store need the persistent kernel");
        tc::gemm_kernel<<<grid, 128, tc::SMEM_BYTES, ctx->stream>>>(mah, mal, mbh, mbl, C, ldc, c_colmajor ? 1 : 0,
                                                                     M, N, ld, ctx->d_status);
    }
    BEM_LAUNCHED(ctx);
    if (ev) {
        const double mn = o.lower ? 0.5 * (double)M * (M + 1) : (double)M * N;  // the lower triangle of C
        ctx->prof_end(prof_cls, ev, 8.0 * mn * K, 8.0 * ((double)M * K + (double)K * N + 2.0 * mn));
    }
    return BEM_OK;
}

static int tc_gemm(bem_ctx* ctx, int M, int N, int K, const float2* A, int64_t lda, const float2* B, int64_t ldb,
                   bool b_rowmajor, float2* C, int64_t ldc, bool c_colmajor, int prof_cls) {
    TcOpts o;
    o.b_rowmajor = b_rowmajor;
    o.c_colmajor = c_colmajor;
    o.prof_cls = prof_cls;
    return tc_gemm_ex(ctx, M, N, K, A, lda, B, ldb, C, ldc, o);
}

static int tc_lu_update(bem_ctx* ctx, void*, int M, int N, int K, const float2* A, int64_t lda, const float2* B,
                        int64_t ldb, float2* C, int64_t ldc) {
    return tc_gemm(ctx, M, N, K, A, lda, B, ldb, true, C, ldc, false, PROF_LU_UPDATE);
}

static int tc_solve_update(bem_ctx* ctx, void*, int M, int N, int K, const float2* A, int64_t lda, const float2* B,
                           int64_t ldb, float2* C, int64_t ldc) {
    return tc_gemm(ctx, M, N, K, A, lda, B, ldb, false, C, ldc, true, PROF_SOLVE_UPDATE);
}

TrailingUpdate<float> tc_update_fp32(bem_ctx* ctx) {
    TrailingUpdate<float> t;
    if (ctx && ctx->use_tc) {
        t.fn = tc_lu_update;
        t.fn_solve = tc_solve_update;
    }
    return t;
}

}  // namespace bem

extern "C" int bem_cgemm_tf32x3(bem_ctx* ctx, int M, int N, int K, const void* A, int64_t lda, const void* B,
                                int64_t ldb, int b_rowmajor, void* C, int64_t ldc, int c_colmajor) {
    if (!ctx || !A || !B || !C) return BEM_ERR_INVALID;
    BEM_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    BEM_TRY_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream));
    BEM_TRY(bem::tc_gemm(ctx, M, N, K, (const float2*)A, lda, (const float2*)B, ldb, b_rowmajor != 0, (float2*)C,
                         ldc, c_colmajor != 0, -1));
    int st = 0;
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(&st, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    BEM_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return st == 0 ? BEM_OK : bem::fail(ctx, st, "tensor-core GEMM: a bounded wait expired");
}
