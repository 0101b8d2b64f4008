// FP64-accurate refinement residual R = B - Z X on the int8 tensor cores
// (Ozaki scheme: error-free slicing into int8 digits, exact int32 products,
// FP64 recombination).
//
// Z' (n x 2n, real, the interleaved complex rows of Z) and X' (2 nrhs x 2n,
// rows 2j: (Re x, -Im x), 2j+1: (Im x, Re x) over k) are scaled per row by a
// power of two so every entry is below 1/2 in magnitude, then split into S
// digits q_s in [-64, 64]:  v = sum_s q_s 2^(-7 s) + r,  |r| <= 2^(-7 S - 1).
// The product keeps the digit pairs with s + t <= S + 1:
//   (Z' X'^T)_ic = 2^(e_i + f_c) sum_{s+t<=S+1} 2^(-7(s+t)) (A_s B_t^T)_ic
// Each A_s B_t^T is exact in int32 (|q q| <= 2^12, 2n <= 2^17 terms); pairs
// with the same s + t share one TMEM accumulator in groups of at most four
// (4 * 2^12 * 2^17 < 2^31).  The epilogue scales by 2^(e_i + f_j - 7(s+t))
// (exact) and subtracts from R in FP64.  With S = 7 the digits carry 48 bits.
// X' may keep fewer digits, Sx <= S (1-based t <= Sx): the refinement rounds
// its iterates to their first Sx digits and keeps the rounded values, so the
// pairs with t > Sx, zero for them, are not computed (slice_cols_kernel
// writes the rounded value back).
//
// The int8 GEMM is the persistent warp-specialised tcgen05 kernel of
// gemm_tc.cu with kind::i8 (M = 128, N = 256, K = 32 per MMA), 4 stages of
// 128-byte K slabs, no multicast.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdint>
#include <vector>

#include "bem_internal.h"
#include "lu_internal.h"
#include "ozaki.h"

namespace bem {
namespace oz {

constexpr int BM = 128, BN = 256, BKB = 128;  // rows, real columns, K bytes per stage
constexpr int STAGES = 4;
constexpr int A_BYTES = BM * BKB;              // 16 KB
constexpr int B_BYTES = BN * BKB;              // 32 KB
constexpr int STAGE_BYTES = A_BYTES + B_BYTES; // 48 KB
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 256;
constexpr uint32_t TMEM_COLS = 512;
constexpr long long WAIT_CYCLES = 2000000000LL;
// Tile raster: groups of GROUP_M row tiles x all column tiles.  A wave of 148
// single-CTA tiles then spans ~16 row tiles x ~9 column tiles, which balances
// the re-reads of the (larger) Z digit rows against those of the X digit rows.
constexpr int GROUP_M = 16;
constexpr int MAXP = 4;  // digit pairs per accumulator group

// 2^k for a normal k, 0 below the normal range (those terms are far below
// FP64 resolution of the residual).
__device__ __forceinline__ double pow2i(int k) {
    if (k < -1022) return 0.0;
    return __longlong_as_double((long long)(min(k, 1023) + 1023) << 52);
}
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
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
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)(1024 >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
    return d;
}
// kind::i8, signed int8 A and B (K-major), int32 accumulate, M = 128, N = 256.
constexpr uint32_t IDESC = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                           ((uint32_t)(BM >> 4) << 24);
__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t accumulate) {
    uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        ::"r"(tmem_d), "l"(a), "l"(b), "r"(IDESC), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
}
__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, int* v) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
          "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
          "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
          "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

struct Group {
    int np;          // digit pairs in this accumulator group (<= MAXP)
    int s[MAXP], t[MAXP];
    int d;           // s + t, common to the group
};
struct Groups {
    int ng;
    Group g[40];
};

// One thread's row of a drained accumulator: 256 int32 columns (128 complex
// RHS columns from jcol0) of TMEM row `row`, scaled by 2^(e_row + f_col - 7d)
// and subtracted from R in FP64.
__device__ __forceinline__ void drain_tile(uint32_t base, double2* __restrict__ R, int64_t ldr, int row, int n,
                                           const int* __restrict__ e_row, const int* __restrict__ f_col, int jcol0,
                                           int nrhs, int d) {
    const int er = row < n ? e_row[row] : 0;
#pragma unroll 1
    for (int ch = 0; ch < BN / 32; ch++) {
        int v[32];
        tmem_ld32(base + ch * 32, v);
        const int j0 = jcol0 + ch * 16;
        if (row < n) {
            // reads of the 16 column segments in flight together, then the writes
            const int nj = min(16, nrhs - j0);
            double2 r[16];
#pragma unroll
            for (int jj = 0; jj < 16; jj++)
                if (jj < nj) r[jj] = R[(int64_t)(j0 + jj) * ldr + row];
#pragma unroll
            for (int jj = 0; jj < 16; jj++)
                if (jj < nj) {
                    const double sc = pow2i(er + f_col[j0 + jj] - 7 * d);
                    r[jj].x -= sc * (double)v[2 * jj];
                    r[jj].y -= sc * (double)v[2 * jj + 1];
                    R[(int64_t)(j0 + jj) * ldr + row] = r[jj];
                }
        }
    }
}

// R[j*ldr + i] -= 2^(e_i + f_j - 7 d) * (A_s B_t^T)[i, 2j + {0,1}] summed over groups.
__global__ void __launch_bounds__(192, 1)
residual_kernel(const __grid_constant__ CUtensorMap tA, const __grid_constant__ CUtensorMap tB,
                const __grid_constant__ Groups G, double2* __restrict__ R, int64_t ldr, const int* __restrict__ e_row,
                const int* __restrict__ f_col, int n, int nrhs, int K2p, unsigned* __restrict__ pace, int pace_epoch,
                int pace_lead, int* status) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t* bars = (uint64_t*)(smem + STAGES * STAGE_BYTES);
    uint64_t* full = bars;
    uint64_t* empty = bars + STAGES;
    uint64_t* tfull = bars + 2 * STAGES;
    uint64_t* tempty = bars + 2 * STAGES + 2;
    uint32_t* tmem_slot = (uint32_t*)(bars + 2 * STAGES + 4);
    __shared__ volatile int abort_flag;
    __shared__ int issued_total, consumed_total;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nk = K2p / BKB;
    const int num_m = (n + BM - 1) / BM, num_n = (2 * nrhs + BN - 1) / BN;
    const int ntiles = num_m * num_n;
    // a CTA owns its tiles (t = blockIdx.x + i gridDim.x) for every digit
    // group, so the FP64 read-modify-writes of one tile never race; the groups
    // are the outer loop so that the CTAs of a wave stream the same digit
    // planes at the same time and share them in L2
    auto unit_tile = [&](int t, int& mt, int& ntl) {
        const int per = GROUP_M * num_n;
        const int gi = t / per, first_m = gi * GROUP_M;
        const int gsz = min(GROUP_M, num_m - first_m);
        const int r = t % per;
        mt = first_m + r % gsz;
        ntl = r / gsz;
    };

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
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            // Pacing: the CTAs of a wave share the digit rows of their tiles
            // through L2 only while they stream the same K slabs at about the
            // same time (K = 2n is ~1000 slabs per digit pair).  Every EPOCH
            // slabs the producer adds one to a grid-wide counter and lets at
            // most LEAD epochs of lead over the grid average build up; the
            // wait is soft (it gives up after PACE_CYCLES), so it cannot hang.
            const int EPOCH = pace_epoch > 0 ? pace_epoch : 1 << 30, LEAD = pace_lead;
            constexpr long long PACE_CYCLES = 200000;
            int np_total = 0;
            for (int gr = 0; gr < G.ng; gr++) np_total += G.g[gr].np;
            const long long max_epochs =
                ((long long)((ntiles + gridDim.x - 1) / gridDim.x) * np_total * nk + EPOCH - 1) / EPOCH;
            long long my_epochs = 0;
            int it = 0;
            for (int gr = 0; gr < G.ng && !abort_flag; gr++)
            for (int u = blockIdx.x; u < ntiles && !abort_flag; u += gridDim.x) {
                int mt, ntl;
                unit_tile(u, mt, ntl);
                const Group& g = G.g[gr];
                for (int p = 0; p < g.np && !abort_flag; p++) {
                    const int ya = g.s[p] * n + mt * BM, yb = g.t[p] * 2 * nrhs + ntl * BN;
                    for (int kt = 0; kt < nk; kt++, it++) {
                        const int s = it % STAGES;
                        if (!mbar_wait(smem_u32(&empty[s]), ((it / STAGES) & 1) ^ 1, status, &abort_flag)) break;
                        unsigned char* st = smem + s * STAGE_BYTES;
                        const uint32_t fb = smem_u32(&full[s]);
                        mbar_expect_tx(fb, STAGE_BYTES);
                        tma_load_2d(smem_u32(st), &tA, kt * BKB, ya, fb);
                        tma_load_2d(smem_u32(st + A_BYTES), &tB, kt * BKB, yb, fb);
                        issued_total = it + 1;
                        if ((it + 1) % EPOCH == 0) {
                            my_epochs++;
                            atomicAdd(pace, 1u);
                            const long long t0 = clock64();
                            while (!abort_flag && clock64() - t0 < PACE_CYCLES) {
                                const long long tot = *(volatile unsigned*)pace;
                                if (my_epochs * gridDim.x <= tot + (long long)LEAD * gridDim.x) break;
                                __nanosleep(256);
                            }
                        }
                    }
                }
            }
            // finished: count as at the end, so the others are not held back
            if (max_epochs > my_epochs) atomicAdd(pace, (unsigned)(max_epochs - my_epochs));
        }
    } else if (warp == 1) {
        if (lane == 0) {
            int it = 0, lt = 0;
            bool stop = false;
            for (int gr = 0; gr < G.ng && !stop; gr++)
            for (int u = blockIdx.x; u < ntiles && !stop; u += gridDim.x, lt++) {
                const Group& g = G.g[gr];
                const int b = lt & 1;
                if (!mbar_wait(smem_u32(&tempty[b]), ((lt >> 1) & 1) ^ 1, status, &abort_flag)) {
                    stop = true;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t acc = tmem + (uint32_t)(b * 256);
                bool ok = true;
                for (int p = 0; p < g.np && ok; p++) {
                    for (int kt = 0; kt < nk; kt++, it++) {
                        const int s = it % STAGES;
                        if (!mbar_wait(smem_u32(&full[s]), (it / STAGES) & 1, status, &abort_flag)) {
                            ok = false;
                            break;
                        }
                        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                        unsigned char* st = smem + s * STAGE_BYTES;
                        const uint32_t a0 = smem_u32(st), b0 = smem_u32(st + A_BYTES);
#pragma unroll
                        for (int ks = 0; ks < BKB / 32; ks++) {
                            const uint32_t off = ks * 32;
                            mma_i8(acc, smem_desc(a0 + off), smem_desc(b0 + off),
                                   (p > 0 || kt > 0 || ks > 0) ? 1u : 0u);
                        }
                        mma_commit(smem_u32(&empty[s]));
                        consumed_total = it + 1;
                    }
                }
                mma_commit(smem_u32(&tfull[b]));
                if (!ok) stop = true;
            }
        }
    } else {
        const int q = warp & 3;
        // R of the next tile is prefetched into L2 while the current one is
        // multiplied (one column segment of 128 rows per thread)
        auto prefetch_r = [&](int u) {
            if (u >= ntiles) return;
            int mt, ntl;
            unit_tile(u, mt, ntl);
            const int j = ntl * (BN / 2) + q * 32 + lane, r0 = mt * BM;
            if (j >= nrhs || r0 >= n) return;
            const char* p = reinterpret_cast<const char*>(&R[(int64_t)j * ldr + r0]);
            const int bytes = min(BM, n - r0) * (int)sizeof(double2);
            for (int o = 0; o < bytes; o += 128) asm volatile("prefetch.global.L2 [%0];" ::"l"(p + o));
        };
        prefetch_r(blockIdx.x);
        int lt = 0;
        bool stop = false;
        for (int gr = 0; gr < G.ng && !stop; gr++)
        for (int u = blockIdx.x; u < ntiles; u += gridDim.x, lt++) {
            prefetch_r(u + gridDim.x);
            const int b = lt & 1;
            bool ok = mbar_wait(smem_u32(&tfull[b]), (lt >> 1) & 1, status, &abort_flag);
            ok = __all_sync(0xffffffffu, ok);
            if (!ok) {
                stop = true;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            int mt, ntl;
            unit_tile(u, mt, ntl);
            const int d = G.g[gr].d;
            const int row = mt * BM + q * 32 + lane;
            const uint32_t base = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * 256);
            drain_tile(base, R, ldr, row, n, e_row, f_col, ntl * (BN / 2), nrhs, d);
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&tempty[b]));
        }
    }
    __syncwarp();
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
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
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
    }
}

// ---------------------------------------------------------------- slicing
// e[i] = ilogb(max_k |Z'[i,k]|) + 2 (so |Z'[i,k] 2^-e| < 1/2); 0 for a zero row.
__global__ void row_exp_kernel(const double2* __restrict__ Z, int64_t ldz, int n, int* __restrict__ e) {
    __shared__ double s[256];
    const double2* row = Z + (int64_t)blockIdx.x * ldz;
    double m = 0.0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) m = fmax(m, fmax(fabs(row[k].x), fabs(row[k].y)));
    s[threadIdx.x] = m;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) s[threadIdx.x] = fmax(s[threadIdx.x], s[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) e[blockIdx.x] = s[0] > 0.0 ? ilogb(s[0]) + 2 : 0;
}

// The right-hand operand: X itself (complex128), or a refinement correction
// held as complex64 D with a per-column FP64 scale, X[:, j] = scale[j] D[:, j]
// (the product rounded to FP64, as the refinement adds it to the iterate).
struct ColSrc {
    const double2* X;
    const float2* D;
    const double* scale;
    int64_t ld;
    __device__ __forceinline__ double2 get(int j, int k) const {
        if (X) return X[(int64_t)j * ld + k];
        const double sc = scale[j];
        const float2 d = D[(int64_t)j * ld + k];
        return make_double2(sc * (double)d.x, sc * (double)d.y);
    }
};

// f[j] for column j of X (column-major): both X' rows 2j, 2j+1 hold the same
// magnitudes, so one exponent per complex column.
__global__ void col_exp_kernel(ColSrc src, int n, int* __restrict__ f) {
    __shared__ double s[256];
    double m = 0.0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const double2 v = src.get(blockIdx.x, k);
        m = fmax(m, fmax(fabs(v.x), fabs(v.y)));
    }
    s[threadIdx.x] = m;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) s[threadIdx.x] = fmax(s[threadIdx.x], s[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) f[blockIdx.x] = s[0] > 0.0 ? ilogb(s[0]) + 2 : 0;
}

__device__ __forceinline__ void digits(double v, int8_t* q) {
#pragma unroll
    for (int s = 0; s < S_MAX; s++) {
        double t = v * 128.0;
        double r = rint(t);
        q[s] = (int8_t)(int)r;
        v = t - r;
    }
}

// A digit planes: A[s][i][k'] int8, k' = 2k + {0: Re, 1: Im}, row pitch ldk bytes.
__global__ void slice_rows_kernel(const double2* __restrict__ Z, int64_t ldz, int n, const int* __restrict__ e,
                                  int8_t* __restrict__ A, int64_t ldk, int64_t plane, int S) {
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t kc = ldk / 2;  // complex slots per row (zero padded)
    if (t >= (int64_t)n * kc) return;
    const int i = (int)(t / kc), k = (int)(t % kc);
    double2 z = k < n ? Z[(int64_t)i * ldz + k] : make_double2(0.0, 0.0);
    const int ex = e[i];
    int8_t qr[S_MAX], qi[S_MAX];
    const double sc = pow2i(-ex);
    digits(z.x * sc, qr);
    digits(z.y * sc, qi);
    for (int s = 0; s < S; s++) {
        char2 c;
        c.x = qr[s];
        c.y = qi[s];
        reinterpret_cast<char2*>(A + s * plane + (int64_t)i * ldk)[k] = c;
    }
}

// B digit planes: B[t][2j + p][k'] for X' rows (Re, -Im) / (Im, Re).
// fix (optional): the value the S digits represent, x~ = 2^ex sum_s q_s
// 128^-(s+1) (exact in FP64 for S <= 7: 49 bits), replaces x there (src.X)
// or corrects it (src.D: fix += x~ - x).
__global__ void slice_cols_kernel(ColSrc src, int n, int nrhs, const int* __restrict__ f, int8_t* __restrict__ B,
                                  int64_t ldk, int64_t plane, int S, double2* __restrict__ fix, int64_t ldfix) {
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t kc = ldk / 2;
    if (t >= (int64_t)nrhs * kc) return;
    const int j = (int)(t / kc), k = (int)(t % kc);
    double2 x = k < n ? src.get(j, k) : make_double2(0.0, 0.0);
    const int ex = f[j];
    int8_t qr[S_MAX], qi[S_MAX];
    const double sc = pow2i(-ex);
    digits(x.x * sc, qr);
    digits(x.y * sc, qi);
    if (fix && k < n) {
        double rr = 0.0, ri = 0.0;
        for (int s = S - 1; s >= 0; s--) {  // Horner in base 128: exact
            rr = (rr + (double)qr[s]) * (1.0 / 128.0);
            ri = (ri + (double)qi[s]) * (1.0 / 128.0);
        }
        const double up = pow2i(ex);
        rr *= up;
        ri *= up;
        double2* p = fix + (int64_t)j * ldfix + k;
        if (src.X) {
            *p = make_double2(rr, ri);
        } else {
            const double2 v = *p;
            *p = make_double2(v.x + (rr - x.x), v.y + (ri - x.y));
        }
    }
    for (int s = 0; s < S; s++) {
        char2 r0, r1;
        r0.x = qr[s];
        r0.y = (int8_t)(-qi[s]);
        r1.x = qi[s];
        r1.y = qr[s];
        reinterpret_cast<char2*>(B + s * plane + (int64_t)(2 * j) * ldk)[k] = r0;
        reinterpret_cast<char2*>(B + s * plane + (int64_t)(2 * j + 1) * ldk)[k] = r1;
    }
}

}  // namespace oz

// ---------------------------------------------------------------- host side
static PFN_cuTensorMapEncodeTiled_v12000 g_encode_i8 = nullptr;

static int encode_i8(bem_ctx* ctx, CUtensorMap* map, void* base, int64_t rows, int64_t ldk, int box_rows) {
    if (!g_encode_i8) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        BEM_TRY_CUDA(ctx, cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !fn) return fail(ctx, BEM_ERR_CUDA, "cuTensorMapEncodeTiled missing");
        g_encode_i8 = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    }
    cuuint64_t dims[2] = {(cuuint64_t)ldk, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)ldk};
    cuuint32_t box[2] = {(cuuint32_t)oz::BKB, (cuuint32_t)box_rows};
    cuuint32_t es[2] = {1, 1};
    CUresult r = g_encode_i8(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, base, dims, strides, box, es,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(ctx, BEM_ERR_CUDA, "cuTensorMapEncodeTiled (int8) failed (%d)", (int)r);
    return BEM_OK;
}

size_t ozaki_z_bytes(int n, int S) {
    int64_t ldk = ((int64_t)2 * n + oz::BKB - 1) / oz::BKB * oz::BKB;
    return (size_t)S * n * ldk + 256 + (size_t)n * sizeof(int);
}

int ozaki_prepare_z(bem_ctx* ctx, OzakiZ* oz_, const double2* Z, int64_t ldz, int n, int S) {
    if (S < 2 || S > oz::S_MAX) return fail(ctx, BEM_ERR_INVALID, "ozaki digits %d", S);
    oz_->n = n;
    oz_->S = S;
    oz_->ldk = ((int64_t)2 * n + oz::BKB - 1) / oz::BKB * oz::BKB;
    oz_->plane = (int64_t)n * oz_->ldk;
    size_t bytes = (size_t)S * oz_->plane;
    oz_->device = ctx->device;
    oz_->owner = ctx;
    oz_->A = (int8_t*)devmem_alloc(ctx->device, bytes, ctx);
    oz_->e = oz_->A ? (int*)devmem_alloc(ctx->device, (size_t)n * sizeof(int), ctx) : nullptr;
    if (!oz_->A || !oz_->e) {
        ozaki_free(oz_);
        return fail(ctx, BEM_ERR_OOM, "ozaki digit planes (%zu bytes)", bytes);
    }
    oz::row_exp_kernel<<<n, 256, 0, ctx->stream>>>(Z, ldz, n, oz_->e);
    BEM_LAUNCHED(ctx);
    int64_t tot = (int64_t)n * (oz_->ldk / 2);
    oz::slice_rows_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, ctx->stream>>>(Z, ldz, n, oz_->e, oz_->A, oz_->ldk,
                                                                                 oz_->plane, S);
    BEM_LAUNCHED(ctx);
    return BEM_OK;
}

void ozaki_free(OzakiZ* oz_) {
    devmem_free(oz_->device, oz_->A, (size_t)oz_->S * oz_->plane, oz_->owner);
    devmem_free(oz_->device, oz_->e, (size_t)oz_->n * sizeof(int), oz_->owner);
    oz_->A = nullptr;
    oz_->e = nullptr;
}

// R -= Z X with the first S digits of Z and the first Sx <= S of X (S <= the
// digits of Z): the digit pairs s + t <= S - 1 (0-based) with t < Sx.  fix:
// see slice_cols_kernel.
static int ozaki_apply(bem_ctx* ctx, const OzakiZ* oz_, oz::ColSrc src, double2* R, int64_t ldr, int nrhs, int S,
                       int Sx, double2* fix, int64_t ldfix) {
    const int n = oz_->n;
    if (S < 2 || S > oz_->S) return fail(ctx, BEM_ERR_INVALID, "ozaki residual: %d digits of %d", S, oz_->S);
    if (Sx < 1 || Sx > S || (fix && Sx > 7))
        return fail(ctx, BEM_ERR_INVALID, "ozaki residual: %d digits of X for %d of Z", Sx, S);
    const int64_t ldk = oz_->ldk;
    const int64_t bplane = (int64_t)2 * nrhs * ldk;
    size_t need = (size_t)Sx * bplane + (size_t)nrhs * sizeof(int) + 512;
    if (need > ctx->oz_bytes) {
        if (ctx->oz_buf) {
            BEM_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            cudaFree(ctx->oz_buf);
        }
        ctx->oz_buf = nullptr;
        ctx->oz_bytes = 0;
        if (cudaMalloc(&ctx->oz_buf, need) != cudaSuccess) {
            cudaGetLastError();
            ctx->oz_buf = nullptr;
            return fail(ctx, BEM_ERR_OOM, "ozaki residual workspace (%zu bytes)", need);
        }
        ctx->oz_bytes = need;
    }
    int8_t* Bd = (int8_t*)ctx->oz_buf;
    int* f = (int*)((char*)ctx->oz_buf + (((size_t)Sx * bplane + 255) & ~(size_t)255));
    cudaEvent_t ev = ctx->prof_begin(PROF_RESIDUAL);
    oz::col_exp_kernel<<<nrhs, 256, 0, ctx->stream>>>(src, n, f);
    BEM_LAUNCHED(ctx);
    int64_t tot = (int64_t)nrhs * (ldk / 2);
    oz::slice_cols_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, ctx->stream>>>(src, n, nrhs, f, Bd, ldk, bplane,
                                                                                  Sx, fix, ldfix);
    BEM_LAUNCHED(ctx);
    CUtensorMap tA, tB;
    BEM_TRY(encode_i8(ctx, &tA, oz_->A, (int64_t)oz_->S * n, ldk, oz::BM));
    BEM_TRY(encode_i8(ctx, &tB, Bd, (int64_t)Sx * 2 * nrhs, ldk, oz::BN));
    // digit pairs s + t <= S + 1 (1-based), grouped by d = s + t, <= MAXP per group
    // int32 safety: maxp pairs of |q q| <= 2^12 over ldk terms stay below 2^31
    const int maxp = (int)std::min<int64_t>(oz::MAXP, ((int64_t)1 << 31) / ((int64_t)4096 * ldk + 1));
    if (maxp < 1) return fail(ctx, BEM_ERR_INVALID, "ozaki residual: n = %d too large for int32 accumulation", n);
    oz::Groups G{};
    for (int d = 2; d <= S + 1; d++) {
        oz::Group cur{};
        cur.d = d;
        for (int s = 1; s < d; s++) {
            int t = d - s;
            if (s > S || t > Sx) continue;
            cur.s[cur.np] = s - 1;
            cur.t[cur.np] = t - 1;
            if (++cur.np == maxp) {
                G.g[G.ng++] = cur;
                cur.np = 0;
            }
        }
        if (cur.np) G.g[G.ng++] = cur;
    }
    if (!ctx->oz_attr) {
        BEM_TRY_CUDA(ctx, cudaFuncSetAttribute(oz::residual_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               oz::SMEM_BYTES));
        ctx->oz_attr = true;
    }
    const int ntiles = ((n + oz::BM - 1) / oz::BM) * ((2 * nrhs + oz::BN - 1) / oz::BN);
    const int grid = std::min(ntiles, ctx->sm_count);
    unsigned* pace = (unsigned*)(ctx->d_status + 32);  // a spare word of the context's status block
    BEM_TRY_CUDA(ctx, cudaMemsetAsync(pace, 0, sizeof(unsigned), ctx->stream));
    oz::residual_kernel<<<grid, 192, oz::SMEM_BYTES, ctx->stream>>>(tA, tB, G, R, ldr, oz_->e, f, n, nrhs,
                                                                    (int)ldk, pace, ctx->oz_pace_epoch,
                                                                    ctx->oz_pace_lead, ctx->d_status);
    BEM_LAUNCHED(ctx);
    if (ev) {
        // int8 digit-pair products (2 M N K each, M = n, N = 2 nrhs, K = 2 n);
        // bytes: the digit planes of Z and X once, R read and written once
        int pairs = 0;
        for (int i = 0; i < G.ng; i++) pairs += G.g[i].np;
        double ops = (double)pairs * 2.0 * n * (2.0 * nrhs) * (2.0 * n);
        double bytes = (double)S * n * 2.0 * n + (double)Sx * 2.0 * nrhs * 2.0 * n + 32.0 * n * (double)nrhs;
        ctx->prof_end(PROF_RESIDUAL, ev, ops, bytes);
    }
    return BEM_OK;
}

// R -= Z X (R already holds B).  X, R: column-major n x nrhs complex128.
int ozaki_residual(bem_ctx* ctx, const OzakiZ* oz_, const double2* X, int64_t ldx, double2* R, int64_t ldr,
                   int nrhs, int x_digits, double2* round_x) {
    oz::ColSrc src{X, nullptr, nullptr, ldx};
    const bool rnd = x_digits > 0 && x_digits < oz_->S && round_x == X;
    return ozaki_apply(ctx, oz_, src, R, ldr, nrhs, oz_->S, rnd ? x_digits : oz_->S, rnd ? round_x : nullptr, ldx);
}

// R -= Z (scale D): the residual of the next refinement iterate from the
// current one (r_{k+1} = r_k - Z d_k), with `digits` digits for the correction
// (it is small against the iterate, so fewer digits reach the same absolute
// accuracy).
int ozaki_residual_update(bem_ctx* ctx, const OzakiZ* oz_, const float2* D, int64_t ldd, const double* scale,
                          double2* R, int64_t ldr, int nrhs, int digits, int d_digits, double2* fix_x, int64_t ldfix) {
    oz::ColSrc src{nullptr, D, scale, ldd};
    const bool rnd = d_digits > 0 && d_digits < digits && fix_x;
    return ozaki_apply(ctx, oz_, src, R, ldr, nrhs, digits, rnd ? d_digits : digits, rnd ? fix_x : nullptr, ldfix);
}

}  // namespace bem
