// Plane-wave right-hand sides, far field and Mueller reduction on the device.
//
// rhs_kernel       -- compute_rhs_planewave (rhs.cpp:6-64) for a batch of
//                     orientations; par and perp share the phase.
// farfield_kernel  -- farfield_batch_kernel (farfield.cu:100-262) for both
//                     polarisations of an orientation at once, with the
//                     S-matrix / Mueller epilogue of main.cpp:811-845 and
//                     amplitude_to_mueller (farfield.cu:464-508) fused.
// mueller_sum      -- deterministic weighted sum over orientations.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "bem_internal.h"

namespace bem {

#define INV4PI_FF 0.079577471545947667884

struct RhsArgs {
    DevHalf h;
    int N, Nq, n_orient;
    double kr, ki, eta;
    const double* RT;  // n_orient * 9, row-major R^T
    const double* E0;  // optional explicit (E0, k_hat) for one wave
    double2* B;
    int64_t ldb;
};

// One thread per (RWG n, orientation o): both polarisations.
__global__ void rhs_kernel(RhsArgs a) {
    int n = blockIdx.x * blockDim.x + threadIdx.x;
    int o = blockIdx.y;
    if (n >= a.N || o >= a.n_orient) return;
    double kh[3], ep[3][3];
    int npol;
    if (a.E0) {
        // explicit single wave: E0 = a.E0[0..2], k_hat = a.E0[3..5]
        npol = 1;
        for (int i = 0; i < 3; i++) ep[0][i] = a.E0[i], kh[i] = a.E0[3 + i];
    } else {
        npol = 2;
        const double* R = a.RT + 9 * o;
        for (int i = 0; i < 3; i++) {
            kh[i] = R[3 * i + 2];
            ep[0][i] = R[3 * i + 0];  // R^T x
            ep[1][i] = R[3 * i + 1];  // R^T y
        }
    }
    double H[2][3];
    for (int p = 0; p < npol; p++) {
        // H0 = k_hat x E0 / eta
        H[p][0] = (kh[1] * ep[p][2] - kh[2] * ep[p][1]) * (1.0 / a.eta);
        H[p][1] = (kh[2] * ep[p][0] - kh[0] * ep[p][2]) * (1.0 / a.eta);
        H[p][2] = (kh[0] * ep[p][1] - kh[1] * ep[p][0]) * (1.0 / a.eta);
    }
    double bE[2][2] = {{0, 0}, {0, 0}}, bH[2][2] = {{0, 0}, {0, 0}};
    for (int h = 0; h < 2; h++) {
        double sE[2][2] = {{0, 0}, {0, 0}}, sH[2][2] = {{0, 0}, {0, 0}};
        for (int q = 0; q < a.Nq; q++) {
            size_t i = ((size_t)(h * a.N + n)) * a.Nq + q;
            double px = a.h.px[i], py = a.h.py[i], pz = a.h.pz[i];
            double fx = a.h.fx[i], fy = a.h.fy[i], fz = a.h.fz[i];
            double jw = a.h.jw[i];
            double s = kh[0] * px + kh[1] * py + kh[2] * pz;
            double sn, cs;
            sincos(a.kr * s, &sn, &cs);
            double ea = exp(-a.ki * s);
            double phr = ea * cs, phi = ea * sn;
            for (int p = 0; p < npol; p++) {
                double fe = fx * ep[p][0] + fy * ep[p][1] + fz * ep[p][2];
                double fh = fx * H[p][0] + fy * H[p][1] + fz * H[p][2];
                sE[p][0] += fe * phr * jw;
                sE[p][1] += fe * phi * jw;
                sH[p][0] += fh * phr * jw;
                sH[p][1] += fh * phi * jw;
            }
        }
        for (int p = 0; p < npol; p++) {
            bE[p][0] += sE[p][0], bE[p][1] += sE[p][1];
            bH[p][0] += sH[p][0], bH[p][1] += sH[p][1];
        }
    }
    for (int p = 0; p < npol; p++) {
        double2* col = a.B + (int64_t)(npol * o + p) * a.ldb;
        col[n] = make_double2(bE[p][0], bE[p][1]);
        col[a.N + n] = make_double2(bH[p][0], bH[p][1]);
    }
}

int rhs_dev(bem_ctx* ctx, const bem_geom* g, double k_re, double k_im, double eta,
            const double* RT_host, const double* E0_host, const double* khat_host, int n_orient,
            void* B, int64_t ldb) {
    if (!g || !B || ldb < 2 * g->N || n_orient < 1 || !(eta > 0))
        return fail(ctx, BEM_ERR_INVALID, "bad rhs arguments");
    BEM_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    size_t bytes = RT_host ? (size_t)n_orient * 9 * 8 : 6 * 8;
    BEM_TRY(ctx->ensure_ws(bytes));
    std::vector<double> tmp(6);
    const double* src = RT_host;
    if (!RT_host) {
        for (int i = 0; i < 3; i++) tmp[i] = E0_host[i], tmp[3 + i] = khat_host[i];
        src = tmp.data();
    }
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(ctx->ws, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
    RhsArgs a;
    a.h = g->half;
    a.N = g->N;
    a.Nq = g->Nq;
    a.n_orient = RT_host ? n_orient : 1;
    a.kr = k_re;
    a.ki = k_im;
    a.eta = eta;
    a.RT = RT_host ? (const double*)ctx->ws : nullptr;
    a.E0 = RT_host ? nullptr : (const double*)ctx->ws;
    a.B = (double2*)B;
    a.ldb = ldb;
    dim3 grid((g->N + 127) / 128, a.n_orient);
    rhs_kernel<<<grid, 128, 0, ctx->stream>>>(a);
    BEM_LAUNCHED(ctx);
    // the workspace is reused by later calls: finish before returning
    BEM_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return BEM_OK;
}

// ------------------------------------------------------------- far field
struct FFArgs {
    DevHalf h;
    int N, Nq, n_orient, ndir, n_calls;
    double kr, ki, eta;
    // coefficients of call c: J at cJ + c*cs, M at cM + c*cs
    const double2* cJ;
    const double2* cM;
    int64_t cs;
    // directions: rhat (n_orient*ndir*3) or generated from RT and theta
    const double* rhat;
    const double* RT;     // n_orient*9
    const double* theta;  // ndir
    // outputs
    double2* Fv;          // n_calls*ndir*3 (optional)
    double* Mo;           // n_orient*16*ndir: w_o M_o / |k|^2 (optional)
    const double* w;      // n_orient
    int gamma_mirror;
};

// theta_d = pi d / (ndir - 1) (main.cpp:331-333) unless an array is given
__device__ __forceinline__ double theta_of(const FFArgs& a, int d) {
    return a.theta ? a.theta[d] : (a.ndir > 1 ? M_PI * d / (a.ndir - 1) : 0.0);
}

// Far-field vectors of both polarisations from the accumulated J and M
// sums, then the S matrix and the weighted Mueller matrix of the direction
// (main.cpp:785-845, amplitude_to_mueller farfield.cu:464-508).
__device__ void ff_epilogue(const FFArgs& a, int o, int d, const double* r, double (*acc)[2]) {
    // F = -ik/(4 pi) (eta (J - r (r.J)) - r x M)   (sM = -1)
    const double pfr = a.ki * INV4PI_FF, pfi = -a.kr * INV4PI_FF;
    double F[2][3][2];
    for (int pol = 0; pol < 2; pol++) {
        double (*J)[2] = &acc[6 * pol];
        double (*M)[2] = &acc[6 * pol + 3];
        double rdJ[2] = {r[0] * J[0][0] + r[1] * J[1][0] + r[2] * J[2][0],
                         r[0] * J[0][1] + r[1] * J[1][1] + r[2] * J[2][1]};
        double mc[3][2];
        for (int c = 0; c < 2; c++) {
            mc[0][c] = r[1] * M[2][c] - r[2] * M[1][c];
            mc[1][c] = r[2] * M[0][c] - r[0] * M[2][c];
            mc[2][c] = r[0] * M[1][c] - r[1] * M[0][c];
        }
        for (int x = 0; x < 3; x++) {
            double vr = a.eta * (J[x][0] - r[x] * rdJ[0]) - mc[x][0];
            double vi = a.eta * (J[x][1] - r[x] * rdJ[1]) - mc[x][1];
            F[pol][x][0] = pfr * vr - pfi * vi;
            F[pol][x][1] = pfr * vi + pfi * vr;
        }
    }
    if (a.Fv) {
        for (int pol = 0; pol < 2; pol++) {
            int c = 2 * o + pol;
            if (c >= a.n_calls) break;
            double2* out = a.Fv + ((size_t)c * a.ndir + d) * 3;
            for (int x = 0; x < 3; x++) out[x] = make_double2(F[pol][x][0], F[pol][x][1]);
        }
    }
    if (a.Mo) {
        // e_par = R^T e_theta_lab, e_perp = R^T y (main.cpp:785-799, 817-831)
        double st, ct;
        sincos(theta_of(a, d), &st, &ct);
        const double* R = a.RT + 9 * o;
        double epa[3], epe[3];
        for (int i = 0; i < 3; i++) {
            epa[i] = R[3 * i] * ct - R[3 * i + 2] * st;
            epe[i] = R[3 * i + 1];
        }
        double S[5][2];  // S1..S4 at index 1..4
        auto proj = [&](int pol, const double* e, double* out) {
            out[0] = F[pol][0][0] * e[0] + F[pol][1][0] * e[1] + F[pol][2][0] * e[2];
            out[1] = F[pol][0][1] * e[0] + F[pol][1][1] * e[1] + F[pol][2][1] * e[2];
        };
        double fp[2];
        // S = -ik F
        const double ikr = a.ki, iki = -a.kr;
        auto mulik = [&](const double* f, double* s) {
            s[0] = ikr * f[0] - iki * f[1];
            s[1] = ikr * f[1] + iki * f[0];
        };
        proj(0, epa, fp); mulik(fp, S[2]);
        proj(0, epe, fp); mulik(fp, S[4]);
        proj(1, epa, fp); mulik(fp, S[3]);
        proj(1, epe, fp); mulik(fp, S[1]);
        auto nrm = [&](int i) { return S[i][0] * S[i][0] + S[i][1] * S[i][1]; };
        // z_ij = S_i conj(S_j)
        auto zr = [&](int i, int j) { return S[i][0] * S[j][0] + S[i][1] * S[j][1]; };
        auto zi = [&](int i, int j) { return S[i][1] * S[j][0] - S[i][0] * S[j][1]; };
        double a1 = nrm(1), a2 = nrm(2), a3 = nrm(3), a4 = nrm(4);
        double M[16];
        M[0] = 0.5 * (a1 + a2 + a3 + a4);
        M[1] = 0.5 * (a2 - a1 + a4 - a3);
        M[2] = zr(2, 3) + zr(1, 4);
        M[3] = zi(2, 3) - zi(1, 4);
        M[4] = 0.5 * (a2 - a1 - a4 + a3);
        M[5] = 0.5 * (a2 + a1 - a4 - a3);
        M[6] = zr(2, 3) - zr(1, 4);
        M[7] = zi(2, 3) + zi(1, 4);
        M[8] = zr(2, 4) + zr(1, 3);
        M[9] = zr(2, 4) - zr(1, 3);
        M[10] = zr(1, 2) + zr(3, 4);
        M[11] = zi(2, 1) + zi(4, 3);
        M[12] = zi(4, 2) + zi(1, 3);
        M[13] = zi(4, 2) - zi(1, 3);
        M[14] = zi(1, 2) - zi(3, 4);
        M[15] = zr(1, 2) - zr(3, 4);
        if (a.gamma_mirror) {
            const int odd[8] = {2, 3, 6, 7, 8, 9, 12, 13};
            for (int i = 0; i < 8; i++) M[odd[i]] = 0.0;
        }
        double k2 = a.kr * a.kr + a.ki * a.ki;
        double wk = a.w[o] / k2;
        for (int i = 0; i < 16; i++) a.Mo[((size_t)o * 16 + i) * a.ndir + d] = wk * M[i];
    }
}

constexpr int FF_LANES = 4;
constexpr int FF_CHUNK = 256;  // points staged per step

// Block: dpb directions x FF_LANES point lanes; grid (direction chunks, orientations).
__global__ void __launch_bounds__(256) farfield_kernel(FFArgs a, int dpb) {
    extern __shared__ double sm[];
    double* s_p = sm;                   // FF_CHUNK * 6 : x y z wfx wfy wfz
    double2* s_c = (double2*)(sm + FF_CHUNK * 6);  // FF_CHUNK * 4 : cJ0 cM0 cJ1 cM1
    const int o = blockIdx.y;
    const int dl = threadIdx.x / FF_LANES, lane = threadIdx.x % FF_LANES;
    const int d = blockIdx.x * dpb + dl;
    const bool active = dl < dpb && d < a.ndir;
    const int c0 = 2 * o, c1 = 2 * o + 1;
    const bool has1 = c1 < a.n_calls;
    double r[3] = {0, 0, 1};
    if (active) {
        if (a.rhat) {
            const double* rr = a.rhat + ((size_t)o * a.ndir + d) * 3;
            r[0] = rr[0], r[1] = rr[1], r[2] = rr[2];
        } else {
            double st, ct;
            sincos(theta_of(a, d), &st, &ct);
            const double* R = a.RT + 9 * o;
            for (int i = 0; i < 3; i++) r[i] = R[3 * i] * st + R[3 * i + 2] * ct;
        }
    }
    double acc[12][2];
    for (int i = 0; i < 12; i++) acc[i][0] = acc[i][1] = 0.0;
    const int P = 2 * a.N * a.Nq;
    for (int base = 0; base < P; base += FF_CHUNK) {
        __syncthreads();
        for (int e = threadIdx.x; e < FF_CHUNK; e += blockDim.x) {
            int p = base + e;
            if (p < P) {
                double w = a.h.jw[p];
                s_p[e * 6 + 0] = a.h.px[p];
                s_p[e * 6 + 1] = a.h.py[p];
                s_p[e * 6 + 2] = a.h.pz[p];
                s_p[e * 6 + 3] = a.h.fx[p] * w;
                s_p[e * 6 + 4] = a.h.fy[p] * w;
                s_p[e * 6 + 5] = a.h.fz[p] * w;
                int n = (p / a.Nq) % a.N;
                s_c[e * 4 + 0] = a.cJ[(int64_t)c0 * a.cs + n];
                s_c[e * 4 + 1] = a.cM[(int64_t)c0 * a.cs + n];
                s_c[e * 4 + 2] = has1 ? a.cJ[(int64_t)c1 * a.cs + n] : make_double2(0, 0);
                s_c[e * 4 + 3] = has1 ? a.cM[(int64_t)c1 * a.cs + n] : make_double2(0, 0);
            } else {
                for (int k = 0; k < 6; k++) s_p[e * 6 + k] = 0.0;
                for (int k = 0; k < 4; k++) s_c[e * 4 + k] = make_double2(0, 0);
            }
        }
        __syncthreads();
        if (!active) continue;
        const int lim = min(FF_CHUNK, P - base);
        for (int e = lane; e < lim; e += FF_LANES) {
            const double* q = s_p + e * 6;
            double rd = r[0] * q[0] + r[1] * q[1] + r[2] * q[2];
            double sn, cs;
            sincos(a.kr * rd, &sn, &cs);
            double ea = a.ki != 0.0 ? exp(a.ki * rd) : 1.0;
            double phr = cs * ea, phi = -sn * ea;  // exp(-i k r.r')
            const double2* cc = s_c + e * 4;
            // u_k = c_k exp(-i k r.r') once per coefficient, then the real
            // weighted basis vector: 40 FP64 operations per point instead of 54
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const double ur = cc[k].x * phr - cc[k].y * phi, ui = cc[k].x * phi + cc[k].y * phr;
#pragma unroll
                for (int x = 0; x < 3; x++) {
                    acc[3 * k + x][0] += q[3 + x] * ur;
                    acc[3 * k + x][1] += q[3 + x] * ui;
                }
            }
        }
    }
    // reduce the FF_LANES lanes of each direction
    __syncthreads();
    double* red = sm;  // blockDim.x * 24
    for (int i = 0; i < 12; i++) {
        red[threadIdx.x * 24 + 2 * i] = acc[i][0];
        red[threadIdx.x * 24 + 2 * i + 1] = acc[i][1];
    }
    __syncthreads();
    if (!active || lane != 0) return;
    for (int l = 1; l < FF_LANES; l++)
        for (int i = 0; i < 24; i++) (&acc[0][0])[i] += red[(threadIdx.x + l) * 24 + i];
    ff_epilogue(a, o, d, r, acc);
}


// The same far field by triangles: the phase exp(-ik rhat.r_q) at a
// triangle's quadrature point is shared by the (up to three) RWG halves on
// it, whose basis is f_h = s_h (u - pi_h) with u = r - c_t.  Per (direction,
// triangle): E0 = sum_q ph_q w_q and Eu = sum_q ph_q w_q u_q, then for each
// coefficient column k the triangle adds alpha_k Eu + gamma_k E0 with
// alpha_k = sum_h c_kh s_h and gamma_k = -sum_h c_kh s_h pi_h (direction
// independent, formed once per block and staged chunk).  One sincos per
// triangle point instead of per RWG-half point, ~4x fewer operations.
constexpr int FT_CHUNK = 64;  // triangles staged per step
constexpr int FF_MAXQ = 13;

__global__ void __launch_bounds__(256) farfield_tri_kernel(FFArgs a, DevTriAsm ta, int nt, const double* coef,
                                                           int dpb) {
    extern __shared__ double sm[];
    double* s_c = sm;                                     // FT_CHUNK * 3 centroids
    double* s_u = s_c + FT_CHUNK * 3;                     // FT_CHUNK * FF_MAXQ * 3
    double* s_w = s_u + FT_CHUNK * FF_MAXQ * 3;           // FT_CHUNK * FF_MAXQ
    double2* s_al = (double2*)(s_w + FT_CHUNK * FF_MAXQ);  // FT_CHUNK * 4
    double2* s_ga = s_al + FT_CHUNK * 4;                  // FT_CHUNK * 4 * 3
    const int o = blockIdx.y, tid = threadIdx.x;
    const int dl = tid / FF_LANES, lane = tid % FF_LANES;
    const int d = blockIdx.x * dpb + dl;
    const bool active = dl < dpb && d < a.ndir;
    const int c0 = 2 * o, c1 = 2 * o + 1;
    const bool has1 = c1 < a.n_calls;
    const int N = a.N, Nq = a.Nq;
    double r[3] = {0, 0, 1};
    if (active) {
        if (a.rhat) {
            const double* rr = a.rhat + ((size_t)o * a.ndir + d) * 3;
            r[0] = rr[0], r[1] = rr[1], r[2] = rr[2];
        } else {
            double st, ct;
            sincos(theta_of(a, d), &st, &ct);
            const double* R = a.RT + 9 * o;
            for (int i = 0; i < 3; i++) r[i] = R[3 * i] * st + R[3 * i + 2] * ct;
        }
    }
    double acc[12][2];
    for (int i = 0; i < 12; i++) acc[i][0] = acc[i][1] = 0.0;
    for (int t0 = 0; t0 < nt; t0 += FT_CHUNK) {
        const int cnt = min(FT_CHUNK, nt - t0);
        __syncthreads();
        for (int e = tid; e < cnt * 3; e += blockDim.x) s_c[e] = ta.c[(size_t)t0 * 3 + e];
        for (int e = tid; e < cnt * Nq; e += blockDim.x) {
            const int tt = e / Nq, q = e % Nq;
            const size_t src = (size_t)(t0 + tt) * Nq + q;
            s_w[tt * FF_MAXQ + q] = ta.jw[src];
            for (int x = 0; x < 3; x++) s_u[(tt * FF_MAXQ + q) * 3 + x] = ta.u[src * 3 + x];
        }
        for (int e = tid; e < cnt * 4; e += blockDim.x) {
            const int tt = e / 4, k = e % 4;  // k: J0 M0 J1 M1
            const double2* src = (k & 1) ? a.cM : a.cJ;
            const int col = k < 2 ? c0 : c1;
            double2 al = make_double2(0, 0), ga[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
            if (k < 2 || has1) {
                for (int j = 0; j < 3; j++) {
                    const int hn = ta.tri_half[(size_t)(t0 + tt) * 3 + j];
                    if (hn < 0) break;
                    const double2 cc = src[(int64_t)col * a.cs + hn % N];
                    const double sg = coef[hn];
                    al.x += cc.x * sg, al.y += cc.y * sg;
                    for (int x = 0; x < 3; x++) {
                        const double sp = sg * ta.pi[(size_t)hn * 3 + x];
                        ga[x].x -= cc.x * sp, ga[x].y -= cc.y * sp;
                    }
                }
            }
            s_al[tt * 4 + k] = al;
            for (int x = 0; x < 3; x++) s_ga[(tt * 4 + k) * 3 + x] = ga[x];
        }
        __syncthreads();
        if (!active) continue;
        for (int tt = lane; tt < cnt; tt += FF_LANES) {
            const double rdc = r[0] * s_c[tt * 3] + r[1] * s_c[tt * 3 + 1] + r[2] * s_c[tt * 3 + 2];
            double E0r = 0, E0i = 0, Eu[3][2] = {{0, 0}, {0, 0}, {0, 0}};
            for (int q = 0; q < Nq; q++) {
                const double* u = &s_u[(tt * FF_MAXQ + q) * 3];
                const double rd = rdc + (r[0] * u[0] + r[1] * u[1] + r[2] * u[2]);
                double sn, cs;
                sincos(a.kr * rd, &sn, &cs);
                const double ea = a.ki != 0.0 ? exp(a.ki * rd) : 1.0;
                const double w = s_w[tt * FF_MAXQ + q];
                const double pr = cs * ea * w, pim = -sn * ea * w;  // exp(-i k rhat.r) w
                E0r += pr, E0i += pim;
#pragma unroll
                for (int x = 0; x < 3; x++) Eu[x][0] += pr * u[x], Eu[x][1] += pim * u[x];
            }
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const double2 al = s_al[tt * 4 + k];
#pragma unroll
                for (int x = 0; x < 3; x++) {
                    const double2 ga = s_ga[(tt * 4 + k) * 3 + x];
                    acc[3 * k + x][0] += al.x * Eu[x][0] - al.y * Eu[x][1] + ga.x * E0r - ga.y * E0i;
                    acc[3 * k + x][1] += al.x * Eu[x][1] + al.y * Eu[x][0] + ga.x * E0i + ga.y * E0r;
                }
            }
        }
    }
    __syncthreads();
    double* red = sm;  // blockDim.x * 24
    for (int i = 0; i < 12; i++) {
        red[tid * 24 + 2 * i] = acc[i][0];
        red[tid * 24 + 2 * i + 1] = acc[i][1];
    }
    __syncthreads();
    if (!active || lane != 0) return;
    for (int l = 1; l < FF_LANES; l++)
        for (int i = 0; i < 24; i++) (&acc[0][0])[i] += red[(tid + l) * 24 + i];
    ff_epilogue(a, o, d, r, acc);
}

// M_avg[i*ndir + d] = sum over o in order of Mo[o][i][d]
__global__ void mueller_sum_kernel(const double* __restrict__ Mo, int n_orient, int nel,
                                   double* __restrict__ out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nel) return;
    double s = 0.0;
    for (int o = 0; o < n_orient; o++) s += Mo[(size_t)o * nel + i];
    out[i] = s;
}

static int launch_ff(bem_ctx* ctx, const bem_geom* g, FFArgs& a) {
    int nchunk = (a.ndir + 63) / 64;
    int dpb = (a.ndir + nchunk - 1) / nchunk;
    int threads = dpb * FF_LANES;
    dim3 grid(nchunk, a.n_orient);
    cudaEvent_t ev = ctx->prof_begin(PROF_FARFIELD);
    if (ctx->ff_kernel == 0) {
        if (g->Nq > FF_MAXQ) return fail(ctx, BEM_ERR_INVALID, "quadrature of %d points (at most %d)", g->Nq, FF_MAXQ);
        size_t smem = std::max((size_t)FT_CHUNK * (3 + FF_MAXQ * 4) * 8 + (size_t)FT_CHUNK * 16 * 16,
                               (size_t)threads * 24 * 8);
        BEM_TRY_CUDA(ctx, cudaFuncSetAttribute(farfield_tri_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)smem));
        farfield_tri_kernel<<<grid, threads, smem, ctx->stream>>>(a, g->tri, g->nt, g->sing_coef, dpb);
    } else {
        size_t smem = std::max((size_t)FF_CHUNK * (6 * 8 + 4 * 16), (size_t)threads * 24 * 8);
        BEM_TRY_CUDA(ctx, cudaFuncSetAttribute(farfield_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)smem));
        farfield_kernel<<<grid, threads, smem, ctx->stream>>>(a, dpb);
    }
    BEM_LAUNCHED(ctx);
    // algorithmic unit: one (orientation, direction, point) term, ~110 flop
    if (ev)
        ctx->prof_end(PROF_FARFIELD, ev, 110.0 * a.n_orient * (double)a.ndir * 2.0 * a.N * a.Nq,
                      (double)a.n_orient * a.ndir * 16 * 8);
    return BEM_OK;
}

int farfield_dev(bem_ctx* ctx, const bem_geom* g, const void* X, int64_t ldx, int n_calls_x,
                 const double* coeffJ_host, const double* coeffM_host, const double* rhat_host,
                 int n_orient, int ndir, double k_re, double k_im, double eta, double* Fv_host) {
    (void)X;
    (void)ldx;
    (void)n_calls_x;
    const int N = g->N;
    int n_calls = 2 * n_orient;
    size_t cb = (size_t)n_calls * N * 16, rb = (size_t)n_orient * ndir * 3 * 8,
           fb = (size_t)n_calls * ndir * 3 * 16;
    size_t off = 0;
    auto take = [&](size_t b) { size_t o = off; off += (b + 255) & ~(size_t)255; return o; };
    size_t oJ = take(cb), oM = take(cb), oR = take(rb), oF = take(fb);
    BEM_TRY(ctx->ensure_ws(off));
    char* ws = (char*)ctx->ws;
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(ws + oJ, coeffJ_host, cb, cudaMemcpyHostToDevice, ctx->stream));
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(ws + oM, coeffM_host, cb, cudaMemcpyHostToDevice, ctx->stream));
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(ws + oR, rhat_host, rb, cudaMemcpyHostToDevice, ctx->stream));
    FFArgs a{};
    a.h = g->half;
    a.N = N;
    a.Nq = g->Nq;
    a.n_orient = n_orient;
    a.ndir = ndir;
    a.n_calls = n_calls;
    a.kr = k_re;
    a.ki = k_im;
    a.eta = eta;
    a.cJ = (const double2*)(ws + oJ);
    a.cM = (const double2*)(ws + oM);
    a.cs = N;
    a.rhat = (const double*)(ws + oR);
    a.Fv = (double2*)(ws + oF);
    BEM_TRY(launch_ff(ctx, g, a));
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(Fv_host, ws + oF, fb, cudaMemcpyDeviceToHost, ctx->stream));
    BEM_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return BEM_OK;
}

int mueller_dev(bem_ctx* ctx, const bem_geom* g, const void* X, int64_t ldx, const double* RT,
                const double* w, int n_orient, double k_re, double k_im, double eta, int ntheta,
                int gamma_mirror, double* M_avg, double* M_orient_dev, double* Fv_host) {
    const int N = g->N;
    size_t rtb = (size_t)n_orient * 9 * 8, wb = (size_t)n_orient * 8, tb = (size_t)ntheta * 8,
           mob = M_orient_dev ? 0 : (size_t)n_orient * 16 * ntheta * 8, mab = (size_t)16 * ntheta * 8,
           fvb = Fv_host ? (size_t)2 * n_orient * ntheta * 3 * 16 : 0;
    size_t off = 0;
    auto take = [&](size_t b) { size_t o = off; off += (b + 255) & ~(size_t)255; return o; };
    size_t oRT = take(rtb), oW = take(wb), oT = take(tb), oMo = take(mob), oMa = take(mab), oFv = take(fvb);
    BEM_TRY(ctx->ensure_ws(off));
    char* ws = (char*)ctx->ws;
    std::vector<double> th(ntheta);
    for (int i = 0; i < ntheta; i++) th[i] = ntheta > 1 ? M_PI * i / (ntheta - 1) : 0.0;
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(ws + oRT, RT, rtb, cudaMemcpyHostToDevice, ctx->stream));
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(ws + oW, w, wb, cudaMemcpyHostToDevice, ctx->stream));
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(ws + oT, th.data(), tb, cudaMemcpyHostToDevice, ctx->stream));
    FFArgs a{};
    a.h = g->half;
    a.N = N;
    a.Nq = g->Nq;
    a.n_orient = n_orient;
    a.ndir = ntheta;
    a.n_calls = 2 * n_orient;
    a.kr = k_re;
    a.ki = k_im;
    a.eta = eta;
    a.cJ = (const double2*)X;
    a.cM = (const double2*)X + N;
    a.cs = ldx;
    a.RT = (const double*)(ws + oRT);
    a.theta = (const double*)(ws + oT);
    a.w = (const double*)(ws + oW);
    a.Mo = M_orient_dev ? M_orient_dev : (double*)(ws + oMo);
    a.gamma_mirror = gamma_mirror;
    a.Fv = Fv_host ? (double2*)(ws + oFv) : nullptr;
    BEM_TRY(launch_ff(ctx, g, a));
    int nel = 16 * ntheta;
    mueller_sum_kernel<<<(nel + 255) / 256, 256, 0, ctx->stream>>>(a.Mo, n_orient, nel, (double*)(ws + oMa));
    BEM_LAUNCHED(ctx);
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(M_avg, ws + oMa, mab, cudaMemcpyDeviceToHost, ctx->stream));
    if (Fv_host) BEM_TRY_CUDA(ctx, cudaMemcpyAsync(Fv_host, ws + oFv, fvb, cudaMemcpyDeviceToHost, ctx->stream));
    BEM_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return BEM_OK;
}

// ---------------------------------------------------- allocation-free variant
// Scratch of bem_farfield_mueller_noalloc: a file-scope device array, so the
// entry point needs no cudaMalloc.  Host code must not use the symbol as an
// address: its device address is looked up per device with
// cudaGetSymbolAddress on the first call there, which should therefore come
// before any stream capture begins.
static __device__ __align__(256) unsigned char g_noalloc_scratch[BEM_NOALLOC_SCRATCH_BYTES];
static void* g_noalloc_dev_ptr[64];
static std::mutex g_noalloc_mu;

static int noalloc_scratch(bem_ctx* ctx, void** out) {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (ctx->device < 0 || ctx->device >= 64) return fail(ctx, BEM_ERR_INVALID, "device ordinal %d", ctx->device);
    if (!g_noalloc_dev_ptr[ctx->device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);  // device is current (cudaSetDevice)
        if (e != cudaSuccess || !p)
            return fail(ctx, BEM_ERR_CUDA, "cudaGetSymbolAddress of the scratch array: %s", cudaGetErrorString(e));
        g_noalloc_dev_ptr[ctx->device] = p;
    }
    *out = g_noalloc_dev_ptr[ctx->device];
    return BEM_OK;
}

int mueller_noalloc(bem_ctx* ctx, const bem_geom* g, const void* X, int64_t ldx, const double* RT,
                    const double* w, int n_orient, double k_re, double k_im, double eta, int ntheta,
                    int gamma_mirror, double* M_out_dev) {
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    size_t rtb = al((size_t)n_orient * 9 * 8), wb = al((size_t)n_orient * 8),
           mob = al((size_t)n_orient * 16 * ntheta * 8);
    if (rtb + wb + mob > (size_t)BEM_NOALLOC_SCRATCH_BYTES)
        return fail(ctx, BEM_ERR_INVALID,
                    "%d orientations x %d angles need %zu bytes of scratch, above the %d-byte maximum of "
                    "bem_farfield_mueller_noalloc; pass fewer orientations per call and add the results",
                    n_orient, ntheta, rtb + wb + mob, (int)BEM_NOALLOC_SCRATCH_BYTES);
    void* base = nullptr;
    BEM_TRY(noalloc_scratch(ctx, &base));
    char* sc = (char*)base;
    double* d_RT = (double*)sc;
    double* d_w = (double*)(sc + rtb);
    double* d_Mo = (double*)(sc + rtb + wb);
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(d_RT, RT, (size_t)n_orient * 9 * 8, cudaMemcpyHostToDevice, ctx->stream));
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(d_w, w, (size_t)n_orient * 8, cudaMemcpyHostToDevice, ctx->stream));
    FFArgs a{};
    a.h = g->half;
    a.N = g->N;
    a.Nq = g->Nq;
    a.n_orient = n_orient;
    a.ndir = ntheta;
    a.n_calls = 2 * n_orient;
    a.kr = k_re;
    a.ki = k_im;
    a.eta = eta;
    a.cJ = (const double2*)X;
    a.cM = (const double2*)X + g->N;
    a.cs = ldx;
    a.RT = d_RT;
    a.theta = nullptr;  // computed in the kernel
    a.w = d_w;
    a.Mo = d_Mo;  // every (o, i, d) entry is written: nothing to clear
    a.gamma_mirror = gamma_mirror;
    BEM_TRY(launch_ff(ctx, g, a));
    int nel = 16 * ntheta;
    mueller_sum_kernel<<<(nel + 255) / 256, 256, 0, ctx->stream>>>(d_Mo, n_orient, nel, M_out_dev);
    BEM_LAUNCHED(ctx);
    return BEM_OK;
}

}  // namespace bem

using namespace bem;

extern "C" {

int bem_farfield_mueller_noalloc(bem_ctx* ctx, const bem_geom* g, const void* X_dev, int64_t ldx,
                                 const double* RT, const double* w, int n_orient, double k_re, double k_im,
                                 double eta_ext, int ntheta, int gamma_mirror, double* M_avg_dev) {
    if (!ctx || !g || !X_dev || !RT || !w || !M_avg_dev || n_orient < 1 || ntheta < 2 || ldx < 2 * g->N)
        return ctx ? fail(ctx, BEM_ERR_INVALID, "bad bem_farfield_mueller_noalloc arguments") : BEM_ERR_INVALID;
    BEM_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    return mueller_noalloc(ctx, g, X_dev, ldx, RT, w, n_orient, k_re, k_im, eta_ext, ntheta, gamma_mirror,
                           M_avg_dev);
}

int bem_rhs_planewave_dev(bem_ctx* ctx, const bem_geom* g, double k_re, double k_im, double eta_ext,
                          const double* RT, int n_orient, void* B_dev, int64_t ldb) {
    if (!ctx || !g || !RT) return BEM_ERR_INVALID;
    return rhs_dev(ctx, g, k_re, k_im, eta_ext, RT, nullptr, nullptr, n_orient, B_dev, ldb);
}

int bem_rhs_planewave(bem_ctx* ctx, const bem_geom* g, double k_re, double k_im, double eta_ext,
                      const double* E0, const double* k_hat, double* b) {
    if (!ctx || !g || !E0 || !k_hat || !b) return BEM_ERR_INVALID;
    BEM_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    void* d = nullptr;
    size_t bytes = (size_t)2 * g->N * 16;
    BEM_TRY_CUDA(ctx, cudaMalloc(&d, bytes));
    int s = rhs_dev(ctx, g, k_re, k_im, eta_ext, nullptr, E0, k_hat, 1, d, 2 * g->N);
    if (s == BEM_OK) s = d2h(ctx, b, d, bytes);
    cudaFree(d);
    return s;
}

int bem_farfield_batch(bem_ctx* ctx, const bem_geom* g, const double* coeffs_J, const double* coeffs_M,
                       const double* r_hats, double k_re, double k_im, double eta_ext, int n_calls,
                       int n_orient, int ndir, double* Fv) {
    if (!ctx || !g || !coeffs_J || !coeffs_M || !r_hats || !Fv || n_orient < 1 || ndir < 1 ||
        n_calls != 2 * n_orient)
        return ctx ? fail(ctx, BEM_ERR_INVALID, "bem_farfield_batch: n_calls must be 2*n_orient")
                   : BEM_ERR_INVALID;
    BEM_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    return farfield_dev(ctx, g, nullptr, 0, n_calls, coeffs_J, coeffs_M, r_hats, n_orient, ndir, k_re,
                        k_im, eta_ext, Fv);
}

int bem_farfield_mueller_dev(bem_ctx* ctx, const bem_geom* g, const void* X_dev, int64_t ldx,
                             const double* RT, const double* w, int n_orient, double k_re, double k_im,
                             double eta_ext, int ntheta, int gamma_mirror, double* M_avg,
                             double* M_orient_dev) {
    if (!ctx || !g || !X_dev || !RT || !w || !M_avg || n_orient < 1 || ntheta < 2 || ldx < 2 * g->N)
        return ctx ? fail(ctx, BEM_ERR_INVALID, "bad bem_farfield_mueller_dev arguments") : BEM_ERR_INVALID;
    BEM_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    return mueller_dev(ctx, g, X_dev, ldx, RT, w, n_orient, k_re, k_im, eta_ext, ntheta, gamma_mirror,
                       M_avg, M_orient_dev);
}

// amplitude_to_mueller (farfield.cu:464-508), host.
int bem_amplitude_to_mueller(const double* S1, const double* S2, const double* S3, const double* S4,
                             int ntheta, double* M) {
    if (!S1 || !S2 || !S3 || !S4 || !M || ntheta < 1) return BEM_ERR_INVALID;
    for (int t = 0; t < ntheta; t++) {
        const double* S[5] = {nullptr, S1 + 2 * t, S2 + 2 * t, S3 + 2 * t, S4 + 2 * t};
        auto nrm = [&](int i) { return S[i][0] * S[i][0] + S[i][1] * S[i][1]; };
        auto zr = [&](int i, int j) { return S[i][0] * S[j][0] + S[i][1] * S[j][1]; };
        auto zi = [&](int i, int j) { return S[i][1] * S[j][0] - S[i][0] * S[j][1]; };
        double a1 = nrm(1), a2 = nrm(2), a3 = nrm(3), a4 = nrm(4);
        double m[16] = {0.5 * (a1 + a2 + a3 + a4), 0.5 * (a2 - a1 + a4 - a3), zr(2, 3) + zr(1, 4),
                        zi(2, 3) - zi(1, 4),       0.5 * (a2 - a1 - a4 + a3), 0.5 * (a2 + a1 - a4 - a3),
                        zr(2, 3) - zr(1, 4),       zi(2, 3) + zi(1, 4),       zr(2, 4) + zr(1, 3),
                        zr(2, 4) - zr(1, 3),       zr(1, 2) + zr(3, 4),       zi(2, 1) + zi(4, 3),
                        zi(4, 2) + zi(1, 3),       zi(4, 2) - zi(1, 3),       zi(1, 2) - zi(3, 4),
                        zr(1, 2) - zr(3, 4)};
        for (int i = 0; i < 16; i++) M[i * ntheta + t] = m[i];
    }
    return BEM_OK;
}

}  // extern "C"
