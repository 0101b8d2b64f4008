// Adjoint contraction of the derivatives of the PMCHWT operator, the
// plane-wave right-hand sides and the far field with respect to the vertex
// coordinates and the interior wavenumber, without forming dZ.
//
// With the forward solutions x_c, the adjoint vectors lambda_c and
// D = diag(I, -I), the operator term of the gradient is
//   -Re sum_c lambda_c^T (dZ/dp) x_c = -Re sum_ij S_ij (dZ D)_ij / dp,
//   S = sym(P D), P = sum_c lambda_c x_c^T,
// because Z D is symmetric (its blocks are the symmetric Galerkin L and K).
// In terms of the N x N blocks of S:
//   Psi = Re sum_mn [WLe L_e + WLi L_i + WK (K_e + K_i)]_mn,
//   WLe = eta_e S11 - S22 / eta_e,  WLi = eta_i S11 - S22 / eta_i,
//   WK = S12 + S21  (all symmetric),
// and dPsi/dp is the operator term up to its sign.  L and K are sums over
// triangle pairs (a, b) of half-pair integrals; with the RWG basis
// f jw = alpha w (r - v_free), alpha = sign l / 2, the area cancels:
//   L_ts = alpha_t alpha_s sum_pq w_p w_q G(R) [ik (r_p - v_Ft).(r_q - v_Fs) - 4i/k]
//   K_ts = alpha_t alpha_s sum_pq w_p w_q g(R) (r_p - v_Ft).((r_p - r_q) x (r_q - v_Fs))
// with G = exp(ikR)/(4 pi R), g = G'(R)/R (the forms of assemble_LK_kernel,
// assembly.cu:14-135, and of this library's assembly).  Psi_ab = Psi_ba for
// symmetric weights, so the derivative with respect to the vertices of a is
// twice the derivative of sum_b Psi_ab through a's points, free vertices and
// edge lengths: grad_pair_kernel, one block per triangle a, analytic.  The
// same-triangle terms (the G_smooth quadrature and the Graglia singular
// correction, apply_singular_corrections, assembly.cu:208-321) are
// differentiated by central differences of the triangle's own term in its 9
// coordinates (grad_self_kernel); their k derivative is analytic.
// grad_rhs_kernel and grad_ff_kernel differentiate the right-hand sides
// (rhs.cpp:6-64) and the far field at fixed coefficients (farfield.cu:100-262)
// per RWG half.  Each kernel writes per-triangle or per-half gradients in the
// triangle's own vertex slots; the host adds them into the vertices.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <vector>

#include "asm_device.cuh"
#include "bem_internal.h"
#include "lu_internal.h"

namespace bem {
namespace {

constexpr int GQ = 13;  // largest quadrature

__device__ __forceinline__ cplx cadd(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ cplx csub(cplx a, cplx b) { return {a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ cplx cscale(cplx a, double s) { return {a.re * s, a.im * s}; }
__device__ __forceinline__ cplx cdiv(cplx a, cplx b) {
    const double d = b.re * b.re + b.im * b.im;
    return {(a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d};
}
__device__ __forceinline__ cplx c2(double2 v) { return {v.x, v.y}; }

// Per-triangle RWG halves: (RWG n or -1, sign, local index of the free vertex)
struct HalfInfo {
    int n[3], sign[3], jf[3];
};

__device__ __forceinline__ HalfInfo load_halves(const int* hinfo, int t) {
    HalfInfo h;
    for (int k = 0; k < 3; k++) {
        h.n[k] = hinfo[(t * 3 + k) * 3];
        h.sign[k] = hinfo[(t * 3 + k) * 3 + 1];
        h.jf[k] = hinfo[(t * 3 + k) * 3 + 2];
    }
    return h;
}

// alpha = sign |v_e1 - v_e2| / 2 with e1, e2 the vertices other than jf
__device__ __forceinline__ double half_alpha(const double* v, int sign, int jf) {
    const int e1 = (jf + 1) % 3, e2 = (jf + 2) % 3;
    const double dx = v[3 * e1] - v[3 * e2], dy = v[3 * e1 + 1] - v[3 * e2 + 1], dz = v[3 * e1 + 2] - v[3 * e2 + 2];
    return 0.5 * sign * sqrt(dx * dx + dy * dy + dz * dz);
}

// adds g * d alpha / d v into gv (9: the triangle's vertices)
__device__ __forceinline__ void alpha_to_vertices(const double* v, int sign, int jf, double g, double* gv) {
    const int e1 = (jf + 1) % 3, e2 = (jf + 2) % 3;
    double d[3];
    for (int c = 0; c < 3; c++) d[c] = v[3 * e1 + c] - v[3 * e2 + c];
    const double l = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    const double f = g * 0.5 * sign / l;
    for (int c = 0; c < 3; c++) {
        gv[3 * e1 + c] += f * d[c];
        gv[3 * e2 + c] -= f * d[c];
    }
}

__device__ __forceinline__ void bary_point(const double* v, double l1, double l2, double* r) {
    const double l0 = 1.0 - l1 - l2;
    for (int c = 0; c < 3; c++) r[c] = (v[c] * l0 + v[3 + c] * l1) + v[6 + c] * l2;
}

struct GradWeights {
    const double2 *WLe, *WLi, *WK, *Weta;  // N x N, row-major, symmetric
    int N;
};

struct PairArgs {
    const double* tv;   // nt x 9
    const int* hinfo;   // nt x 3 x 3
    int nt, Nq;
    TriQ q;
    Medium ke, ki;
    GradWeights W;
    double* gtri;       // nt x 9: d Psi / d (vertices of the triangle), pair terms
    double* sk;         // nt x 2: sum of WLi dL_i/dk_i + WK dK_i/dk_i over the triangle's pairs
    double* seta;       // nt x 2: sum of Weta L_i
};

// Block reduction of `cnt` doubles per thread into out (thread 0 writes).
template <int CNT>
__device__ void block_sum(double* vals, double* smem, double* out) {
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
    for (int i = 0; i < CNT; i++) {
        double v = vals[i];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) smem[wid * CNT + i] = v;
    }
    __syncthreads();
    if (tid < CNT) {
        double s = 0.0;
        for (int w = 0; w < nw; w++) s += smem[w * CNT + tid];
        out[tid] = s;
    }
}

// One block per triangle a; its threads take the triangles b != a.
__global__ void __launch_bounds__(128) grad_pair_kernel(PairArgs a) {
    const int ta = blockIdx.x, tid = threadIdx.x, Nq = a.Nq, N = a.W.N;
    __shared__ double s_va[9], s_rp[GQ][3], s_alpha[3];
    __shared__ double s_red[4 * 13];
    if (tid < 9) s_va[tid] = a.tv[9 * ta + tid];
    __syncthreads();
    const HalfInfo ha = load_halves(a.hinfo, ta);
    if (tid < Nq) bary_point(s_va, a.q.l1[tid], a.q.l2[tid], s_rp[tid]);
    if (tid < 3) s_alpha[tid] = ha.n[tid] >= 0 ? half_alpha(s_va, ha.sign[tid], ha.jf[tid]) : 0.0;
    __syncthreads();

    double gv[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    double gF[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, gal[3] = {0, 0, 0};
    cplx Sk = {0, 0}, Se = {0, 0};
    const Medium med[2] = {a.ke, a.ki};

    for (int tb = tid; tb < a.nt; tb += blockDim.x) {
        if (tb == ta) continue;
        double vb[9];
        for (int j = 0; j < 9; j++) vb[j] = a.tv[9 * tb + j];
        const HalfInfo hb = load_halves(a.hinfo, tb);
        double as[3];
        for (int s = 0; s < 3; s++) as[s] = hb.n[s] >= 0 ? half_alpha(vb, hb.sign[s], hb.jf[s]) : 0.0;
        for (int t = 0; t < 3; t++) {
            const int nt_ = ha.n[t];
            if (nt_ < 0) continue;
            // weights of half t against the halves of b, aggregated over s:
            // sum_s c_ts (r_q - v_Fs) = A r_q - B
            cplx A0 = {0, 0}, A1 = {0, 0}, C = {0, 0}, Ae = {0, 0};
            cplx B0[3], B1[3], D[3], Be[3];
            for (int c = 0; c < 3; c++) B0[c] = B1[c] = D[c] = Be[c] = {0, 0};
            for (int s = 0; s < 3; s++) {
                const int ns = hb.n[s];
                if (ns < 0) continue;
                const double aa = s_alpha[t] * as[s];
                const size_t ix = (size_t)nt_ * N + ns;
                const cplx w0 = cscale(c2(a.W.WLe[ix]), aa), w1 = cscale(c2(a.W.WLi[ix]), aa),
                           wk = cscale(c2(a.W.WK[ix]), aa), we = cscale(c2(a.W.Weta[ix]), aa);
                A0 = cadd(A0, w0), A1 = cadd(A1, w1), C = cadd(C, wk), Ae = cadd(Ae, we);
                const double* vf = vb + 3 * hb.jf[s];
                for (int c = 0; c < 3; c++) {
                    B0[c] = cadd(B0[c], cscale(w0, vf[c]));
                    B1[c] = cadd(B1[c], cscale(w1, vf[c]));
                    D[c] = cadd(D[c], cscale(wk, vf[c]));
                    Be[c] = cadd(Be[c], cscale(we, vf[c]));
                }
            }
            const double* vFt = s_va + 3 * ha.jf[t];
            for (int p = 0; p < Nq; p++) {
                const double rp[3] = {s_rp[p][0], s_rp[p][1], s_rp[p][2]};
                const double u[3] = {rp[0] - vFt[0], rp[1] - vFt[1], rp[2] - vFt[2]};
                double grp[3] = {0, 0, 0};
                for (int q = 0; q < Nq; q++) {
                    double rq[3];
                    bary_point(vb, a.q.l1[q], a.q.l2[q], rq);
                    const double d[3] = {rp[0] - rq[0], rp[1] - rq[1], rp[2] - rq[2]};
                    const double R2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
                    const double invR = rsqrt(R2), R = R2 * invR;
                    const double dh[3] = {d[0] * invR, d[1] * invR, d[2] * invR};
                    const double ww = a.q.w[p] * a.q.w[q];
#pragma unroll
                    for (int e = 0; e < 2; e++) {
                        const Medium k = med[e];
                        double sn, cs;
                        sincos(k.kr * R, &sn, &cs);
                        const double ea = k.ki != 0.0 ? exp(-k.ki * R) : 1.0;
                        const double i4R = INV4PI_D * invR;
                        const cplx G = {ea * cs * i4R, ea * sn * i4R};
                        const cplx ik = {-k.ki, k.kr};
                        const cplx dG = cmul(G, cplx{-k.ki - invR, k.kr});  // G' = G (ik - 1/R)
                        const cplx gc = cscale(dG, invR);
                        // g' = -G (k^2 R^2 + 3 i k R - 3) / R^3
                        const cplx kk = cmul(cplx{k.kr, k.ki}, cplx{k.kr, k.ki});
                        const cplx pg = {kk.re * R2 - 3.0 * k.ki * R - 3.0, kk.im * R2 + 3.0 * k.kr * R};
                        const cplx dgc = cscale(cmul(G, pg), -invR * invR * invR);
                        const double kn = k.kr * k.kr + k.ki * k.ki;
                        const cplx fik = {4.0 * k.ki / kn, 4.0 * k.kr / kn};  // 4i/k
                        const cplx Aw = e ? A1 : A0;
                        const cplx* Bw = e ? B1 : B0;
                        cplx Vt[3], Wt[3];
                        for (int c = 0; c < 3; c++) {
                            Vt[c] = csub(cscale(Aw, rq[c]), Bw[c]);
                            Wt[c] = csub(cscale(C, rq[c]), D[c]);
                        }
                        const cplx uv = cadd(cadd(cscale(Vt[0], u[0]), cscale(Vt[1], u[1])), cscale(Vt[2], u[2]));
                        const cplx QL = csub(cmul(ik, uv), cmul(fik, Aw));
                        cplx dxW[3], Wxu[3];
                        for (int c = 0; c < 3; c++) {
                            const int c1 = (c + 1) % 3, c2_ = (c + 2) % 3;
                            dxW[c] = csub(cscale(Wt[c2_], d[c1]), cscale(Wt[c1], d[c2_]));
                            Wxu[c] = csub(cscale(Wt[c1], u[c2_]), cscale(Wt[c2_], u[c1]));
                        }
                        const cplx tau =
                            cadd(cadd(cscale(dxW[0], u[0]), cscale(dxW[1], u[1])), cscale(dxW[2], u[2]));
                        const cplx fL = cscale(cmul(G, QL), ww), fK = cscale(cmul(gc, tau), ww);
                        gal[t] += fL.re + fK.re;
                        const cplx cd = cscale(cadd(cmul(dG, QL), cmul(dgc, tau)), ww);
                        const cplx Gik = cscale(cmul(G, ik), ww), gcw = cscale(gc, ww);
                        for (int c = 0; c < 3; c++) {
                            const cplx a1 = cmul(Gik, Vt[c]), a2 = cmul(gcw, dxW[c]), a3 = cmul(gcw, Wxu[c]);
                            grp[c] += cd.re * dh[c] + a1.re + a2.re + a3.re;
                            gF[t][c] -= a1.re + a2.re;
                        }
                        if (e == 1) {
                            // d/dk: dG/dk = i R G, d(gc)/dk = -k G
                            const cplx iRG = cmul(cplx{0.0, R}, G);
                            const cplx kn2 = cmul(cplx{k.kr, k.ki}, cplx{k.kr, k.ki});
                            const cplx f4k2 = cdiv(cplx{0.0, 4.0}, kn2);  // 4i/k^2
                            const cplx dQ = cadd(cmul(cplx{0.0, 1.0}, uv), cmul(f4k2, Aw));
                            cplx sk = cadd(cmul(iRG, QL), cmul(G, dQ));
                            sk = csub(sk, cmul(cmul(cplx{k.kr, k.ki}, G), tau));
                            Sk = cadd(Sk, cscale(sk, ww));
                            cplx Ve[3];
                            for (int c = 0; c < 3; c++) Ve[c] = csub(cscale(Ae, rq[c]), Be[c]);
                            const cplx uve =
                                cadd(cadd(cscale(Ve[0], u[0]), cscale(Ve[1], u[1])), cscale(Ve[2], u[2]));
                            Se = cadd(Se, cscale(cmul(G, csub(cmul(ik, uve), cmul(fik, Ae))), ww));
                        }
                    }
                }
                const double l1 = a.q.l1[p], l2 = a.q.l2[p], l0 = 1.0 - l1 - l2;
                for (int c = 0; c < 3; c++) {
                    gv[c] += l0 * grp[c];
                    gv[3 + c] += l1 * grp[c];
                    gv[6 + c] += l2 * grp[c];
                }
            }
        }
    }
    for (int t = 0; t < 3; t++) {
        if (ha.n[t] < 0) continue;
        for (int c = 0; c < 3; c++) gv[3 * ha.jf[t] + c] += gF[t][c];
        alpha_to_vertices(s_va, ha.sign[t], ha.jf[t], gal[t] / s_alpha[t], gv);
    }
    // Psi_ab = Psi_ba: the b-side derivatives are the a-side ones of (b, a)
    double vals[13];
    for (int i = 0; i < 9; i++) vals[i] = 2.0 * gv[i];
    vals[9] = Sk.re, vals[10] = Sk.im, vals[11] = Se.re, vals[12] = Se.im;
    __shared__ double s_out[13];
    block_sum<13>(vals, s_red, s_out);
    __syncthreads();
    if (tid < 9) a.gtri[9 * ta + tid] = s_out[tid];
    if (tid == 0) {
        a.sk[2 * ta] = s_out[9], a.sk[2 * ta + 1] = s_out[10];
        a.seta[2 * ta] = s_out[11], a.seta[2 * ta + 1] = s_out[12];
    }
}

struct SelfArgs {
    const double* tv;
    const int* hinfo;
    int nt, Nq;
    TriQ q;
    Medium ke, ki;
    unsigned flags;
    GradWeights W;
    double* gtri;   // nt x 9 (central differences of the triangle's own term)
    double* sk;     // nt x 4: the k contraction for Re k, then for Im k (complex each)
    double* seta;   // nt x 2
};

// The triangle's own term: Re sum over its ordered half pairs (t, s) and both
// media of W_e(n_t, n_s) times the same-triangle part of L_e(n_t, n_s) -- the
// G_smooth quadrature (assembly kernels with sing = true) plus the Graglia
// correction (singular_fixup_kernel); with want_k / eta also the interior
// medium's k derivative and the Weta contraction.
// The interior wavenumber enters holomorphically everywhere except at the
// coincident points of the literal G_smooth, exp(ik R_s)/(4 pi R_s) -
// 1/(4 pi R_s) at R_s = 1e-15: there the real part is the rounding of
// exp(-Im k R_s) cos(Re k R_s) to 1 (zero, or a step of one unit in the last
// place) and does not follow Im k, while the imaginary part follows Re k.  So
// the k derivative is returned for Re k (skr) and Im k (ski) separately.
__device__ double self_term(const double* v, const HalfInfo& h, const SelfArgs& a, bool extra, cplx* skr, cplx* ski,
                            cplx* se) {
    const int Nq = a.Nq, N = a.W.N;
    double rp[GQ][3];
    for (int p = 0; p < Nq; p++) bary_point(v, a.q.l1[p], a.q.l2[p], rp[p]);
    double al[3];
    for (int t = 0; t < 3; t++) al[t] = h.n[t] >= 0 ? half_alpha(v, h.sign[t], h.jf[t]) : 0.0;
    const double e1x = v[3] - v[0], e1y = v[4] - v[1], e1z = v[5] - v[2];
    const double e2x = v[6] - v[0], e2y = v[7] - v[1], e2z = v[8] - v[2];
    const double nx = e1y * e2z - e1z * e2y, ny = e1z * e2x - e1x * e2z, nz = e1x * e2y - e1y * e2x;
    const double area = 0.5 * sqrt(nx * nx + ny * ny + nz * nz);
    // Graglia P and V at the triangle's points
    double P[GQ], V[GQ][3];
    for (int p = 0; p < Nq; p++) graglia_point(v, a.q.l1[p], a.q.l2[p], a.q, &P[p], V[p]);
    const bool exact = (a.flags & BEM_ASM_GSMOOTH_EXACT) != 0;
    const Medium med[2] = {a.ke, a.ki};
    double psi = 0.0;
    if (extra) *skr = *ski = *se = {0, 0};
    for (int t = 0; t < 3; t++) {
        if (h.n[t] < 0) continue;
        const double* vFt = v + 3 * h.jf[t];
        for (int s = 0; s < 3; s++) {
            if (h.n[s] < 0) continue;
            const double* vFs = v + 3 * h.jf[s];
            const double aa = al[t] * al[s];
            const size_t ix = (size_t)h.n[t] * N + h.n[s];
            // Graglia sums (without the alpha alpha / A factor)
            double sA = 0.0, sB = 0.0;
            for (int p = 0; p < Nq; p++) {
                sA += a.q.w[p] * P[p];
                double dot = 0.0;
                for (int c = 0; c < 3; c++) dot += (rp[p][c] - vFt[c]) * (V[p][c] - vFs[c] * P[p]);
                sB += a.q.w[p] * dot;
            }
            const double SA = 4.0 * aa / area * sA * INV4PI_D, SB = aa / area * sB * INV4PI_D;
            for (int e = 0; e < 2; e++) {
                const Medium k = med[e];
                const cplx ik = {-k.ki, k.kr};
                const double kn = k.kr * k.kr + k.ki * k.ki;
                const cplx iok = {k.ki / kn, k.kr / kn};  // i/k
                cplx Ls = {0, 0}, Lkr = {0, 0}, Lki = {0, 0};
                for (int p = 0; p < Nq; p++)
                    for (int q = 0; q < Nq; q++) {
                        const double d0 = rp[p][0] - rp[q][0], d1 = rp[p][1] - rp[q][1], d2 = rp[p][2] - rp[q][2];
                        const double R2 = fmax(d0 * d0 + d1 * d1 + d2 * d2, 1e-30);
                        const double invR = rsqrt(R2), Rs = R2 * invR;
                        const double i4R = __dmul_rn(INV4PI_D, invR);
                        double sn, cs;
                        sincos(k.kr * Rs, &sn, &cs);
                        const double ea = k.ki != 0.0 ? exp_decay(k.ki * Rs) : 1.0;
                        cplx Gs = {ea * cs * i4R - i4R, ea * sn * i4R};
                        if (exact) Gs = g_smooth_exact(k, p == q ? 0.0 : Rs);
                        double uu = 0.0;
                        for (int c = 0; c < 3; c++) uu += (rp[p][c] - vFt[c]) * (rp[q][c] - vFs[c]);
                        const double ww = a.q.w[p] * a.q.w[q];
                        // G_s (ik u.u' - 4i/k)
                        const cplx Q = {ik.re * uu - 4.0 * iok.re, ik.im * uu - 4.0 * iok.im};
                        const cplx term = cmul(Gs, Q);
                        Ls.re += ww * term.re, Ls.im += ww * term.im;
                        if (extra && e == 1) {
                            // dG_s/dk = i exp(ikR)/(4 pi); d Q/dk = i u.u' + 4i/k^2
                            const cplx dGs = {-ea * sn * INV4PI_D, ea * cs * INV4PI_D};
                            const cplx f4k2 = cdiv(cplx{0.0, 4.0}, cmul(cplx{k.kr, k.ki}, cplx{k.kr, k.ki}));
                            const cplx dQ = {f4k2.re, uu + f4k2.im};
                            const cplx dt = cadd(cmul(dGs, Q), cmul(Gs, dQ));
                            Lkr.re += ww * dt.re, Lkr.im += ww * dt.im;
                            // d/dIm k = i d/dk, except the literal G_s at a coincident point
                            const cplx di = (p == q && !exact) ? cmul(Gs, cmul(cplx{0.0, 1.0}, dQ))
                                                               : cmul(cplx{0.0, 1.0}, dt);
                            Lki.re += ww * di.re, Lki.im += ww * di.im;
                        }
                    }
                // L_e(self) = alpha alpha sum + (-(i/k) SA + ik SB)
                const cplx corr = {-iok.re * SA + ik.re * SB, -iok.im * SA + ik.im * SB};
                const cplx Lself = {aa * Ls.re + corr.re, aa * Ls.im + corr.im};
                const cplx W = c2((e ? a.W.WLi : a.W.WLe)[ix]);
                psi += W.re * Lself.re - W.im * Lself.im;
                if (extra && e == 1) {
                    // d/dk of the correction: (i/k^2) SA + i SB (holomorphic)
                    const cplx ik2 = cdiv(cplx{0.0, 1.0}, cmul(cplx{k.kr, k.ki}, cplx{k.kr, k.ki}));
                    const cplx dcorr = {ik2.re * SA, ik2.im * SA + SB};
                    const cplx dLr = {aa * Lkr.re + dcorr.re, aa * Lkr.im + dcorr.im};
                    const cplx dci = cmul(cplx{0.0, 1.0}, dcorr);
                    const cplx dLi = {aa * Lki.re + dci.re, aa * Lki.im + dci.im};
                    *skr = cadd(*skr, cmul(W, dLr));
                    *ski = cadd(*ski, cmul(W, dLi));
                    *se = cadd(*se, cmul(c2(a.W.Weta[ix]), Lself));
                }
            }
        }
    }
    return psi;
}

// One thread per triangle: central differences of its own term in its 9
// coordinates (step 1e-4 of its longest edge), and the k / eta contractions.
__global__ void __launch_bounds__(64) grad_self_kernel(SelfArgs a) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.nt) return;
    double v[9];
    for (int j = 0; j < 9; j++) v[j] = a.tv[9 * t + j];
    const HalfInfo h = load_halves(a.hinfo, t);
    double lmax = 0.0;
    for (int j = 0; j < 3; j++) {
        const int j1 = (j + 1) % 3;
        const double dx = v[3 * j] - v[3 * j1], dy = v[3 * j + 1] - v[3 * j1 + 1], dz = v[3 * j + 2] - v[3 * j1 + 2];
        lmax = fmax(lmax, sqrt(dx * dx + dy * dy + dz * dz));
    }
    const double hstep = 1e-4 * lmax;
    cplx skr, ski, se;
    self_term(v, h, a, true, &skr, &ski, &se);
    for (int j = 0; j < 9; j++) {
        const double v0 = v[j];
        v[j] = v0 + hstep;
        const double fp = self_term(v, h, a, false, nullptr, nullptr, nullptr);
        v[j] = v0 - hstep;
        const double fm = self_term(v, h, a, false, nullptr, nullptr, nullptr);
        v[j] = v0;
        a.gtri[9 * t + j] = (fp - fm) / (2.0 * hstep);
    }
    a.sk[4 * t] = skr.re, a.sk[4 * t + 1] = skr.im, a.sk[4 * t + 2] = ski.re, a.sk[4 * t + 3] = ski.im;
    a.seta[2 * t] = se.re, a.seta[2 * t + 1] = se.im;
}

struct HalfArgs {
    const double* tv;
    const int* htri;  // (2N) triangle of half h*N+n
    const int* hjf;   // (2N) local free vertex of the half
    int N, Nq;
    TriQ q;
    double kr, ki, eta;
    const double* RT;         // n_orient x 9
    int n_orient;
    const double2* Lam;       // adjoint vectors, column-major n x 2 n_orient
    int64_t ldl;
    double* ghalf;            // 2N x 9
};

// Right-hand sides: Re sum_c lambda_c^T dB_c, per RWG half (thread), with
// B_c[n] = sum_t alpha_t sum_p w_p (r_p - v_Ft).E0_c exp(ik khat_c.r_p) and
// H0_c = khat_c x E0_c / eta in the rows N + n (rhs.cpp:6-64).
__global__ void grad_rhs_kernel(HalfArgs a) {
    const int hn = blockIdx.x * blockDim.x + threadIdx.x;
    if (hn >= 2 * a.N) return;
    const int n = hn % a.N, sign = hn < a.N ? 1 : -1, t = a.htri[hn], jf = a.hjf[hn], Nq = a.Nq;
    double v[9];
    for (int j = 0; j < 9; j++) v[j] = a.tv[9 * t + j];
    const double al = half_alpha(v, sign, jf);
    const double* vF = v + 3 * jf;
    double gv[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, gF[3] = {0, 0, 0}, gal = 0.0;
    double rp[GQ][3];
    for (int p = 0; p < Nq; p++) bary_point(v, a.q.l1[p], a.q.l2[p], rp[p]);
    double grp[GQ][3];
    for (int p = 0; p < Nq; p++) grp[p][0] = grp[p][1] = grp[p][2] = 0.0;
    for (int o = 0; o < a.n_orient; o++) {
        const double* R = a.RT + 9 * o;
        double kh[3], ep[2][3], H[2][3];
        for (int i = 0; i < 3; i++) kh[i] = R[3 * i + 2], ep[0][i] = R[3 * i], ep[1][i] = R[3 * i + 1];
        for (int pl = 0; pl < 2; pl++) {
            H[pl][0] = (kh[1] * ep[pl][2] - kh[2] * ep[pl][1]) / a.eta;
            H[pl][1] = (kh[2] * ep[pl][0] - kh[0] * ep[pl][2]) / a.eta;
            H[pl][2] = (kh[0] * ep[pl][1] - kh[1] * ep[pl][0]) / a.eta;
        }
        cplx Q[3] = {{0, 0}, {0, 0}, {0, 0}};
        for (int pl = 0; pl < 2; pl++) {
            const int c = 2 * o + pl;
            const cplx lj = c2(a.Lam[(int64_t)c * a.ldl + n]), lm = c2(a.Lam[(int64_t)c * a.ldl + a.N + n]);
            for (int i = 0; i < 3; i++) Q[i] = cadd(Q[i], cadd(cscale(lj, ep[pl][i]), cscale(lm, H[pl][i])));
        }
        for (int p = 0; p < Nq; p++) {
            const double s = kh[0] * rp[p][0] + kh[1] * rp[p][1] + kh[2] * rp[p][2];
            double sn, cs;
            sincos(a.kr * s, &sn, &cs);
            const double ea = exp(-a.ki * s);
            const cplx ph = {ea * cs, ea * sn};  // exp(ik s)
            const double u[3] = {rp[p][0] - vF[0], rp[p][1] - vF[1], rp[p][2] - vF[2]};
            const cplx uQ = cadd(cadd(cscale(Q[0], u[0]), cscale(Q[1], u[1])), cscale(Q[2], u[2]));
            const cplx pQ = cmul(ph, uQ);
            const cplx ikp = cmul(cplx{-a.ki, a.kr}, pQ);  // ik phase (u.Q)
            const double w = a.q.w[p];
            for (int i = 0; i < 3; i++) {
                const cplx pq = cmul(ph, Q[i]);
                grp[p][i] += al * w * (pq.re + ikp.re * kh[i]);
                gF[i] -= al * w * pq.re;
            }
            gal += w * pQ.re;
        }
    }
    for (int p = 0; p < Nq; p++) {
        const double l1 = a.q.l1[p], l2 = a.q.l2[p], l0 = 1.0 - l1 - l2;
        for (int c = 0; c < 3; c++) {
            gv[c] += l0 * grp[p][c];
            gv[3 + c] += l1 * grp[p][c];
            gv[6 + c] += l2 * grp[p][c];
        }
    }
    for (int c = 0; c < 3; c++) gv[3 * jf + c] += gF[c];
    alpha_to_vertices(v, sign, jf, gal, gv);
    for (int j = 0; j < 9; j++) a.ghalf[9 * (size_t)hn + j] = gv[j];
}

struct FFArgs2 {
    const double* tv;
    const int* htri;
    const int* hjf;
    int N, Nq;
    TriQ q;
    double kr, ki, eta;
    const double* RT;      // n_orient x 9
    int ntheta, ncols;
    const double2* hp;     // [c][theta][3]: adjoint weight h of the far field
    const double2* rh;     // [c][theta][3]: rhat x h
    const double2* X;      // forward solutions, column-major n x ncols
    int64_t ldx;
    double* ghalf;         // 2N x 9
};

// Far field at fixed coefficients: Re sum_c sum_theta h . dF_c(theta), per
// RWG half (thread), F = -ik/(4 pi) [eta J_perp - rhat x M] with
// J = sum_n x_n sum_t alpha_t sum_p w_p (r_p - v_Ft) exp(-ik rhat.r_p)
// (farfield.cu:100-262); one block walks every column for its halves.
__global__ void __launch_bounds__(32) grad_ff_kernel(FFArgs2 a) {
    extern __shared__ __align__(16) double sm2[];
    double* s_r = sm2;                                          // ntheta * 3 (padded to 16 bytes)
    double2* s_h = (double2*)(sm2 + ((3 * a.ntheta + 1) & ~1));  // ntheta * 3
    double2* s_x = s_h + 3 * a.ntheta;                          // ntheta * 3
    const int hn = blockIdx.x * blockDim.x + threadIdx.x;
    const bool act = hn < 2 * a.N;
    const int n = act ? hn % a.N : 0, sign = hn < a.N ? 1 : -1;
    const int t = act ? a.htri[hn] : 0, jf = act ? a.hjf[hn] : 0, Nq = a.Nq;
    double v[9];
    for (int j = 0; j < 9; j++) v[j] = a.tv[9 * t + j];
    const double al = act ? half_alpha(v, sign, jf) : 0.0;
    const double* vF = v + 3 * jf;
    double rp[GQ][3];
    for (int p = 0; p < Nq; p++) bary_point(v, a.q.l1[p], a.q.l2[p], rp[p]);
    double grp[GQ][3];
    for (int p = 0; p < Nq; p++) grp[p][0] = grp[p][1] = grp[p][2] = 0.0;
    double gF[3] = {0, 0, 0}, gal = 0.0;
    const cplx pk = {a.ki * INV4PI_D, -a.kr * INV4PI_D};  // -ik/(4 pi)
    const cplx mik = {a.ki, -a.kr};                        // -ik
    for (int c = 0; c < a.ncols; c++) {
        const int o = c / 2;
        __syncthreads();
        for (int th = threadIdx.x; th < a.ntheta; th += blockDim.x) {
            const double ang = a.ntheta > 1 ? M_PI * th / (a.ntheta - 1) : 0.0;
            double st, ct;
            sincos(ang, &st, &ct);
            const double* R = a.RT + 9 * o;
            for (int i = 0; i < 3; i++) s_r[3 * th + i] = R[3 * i] * st + R[3 * i + 2] * ct;
            for (int i = 0; i < 3; i++) {
                s_h[3 * th + i] = a.hp[((size_t)c * a.ntheta + th) * 3 + i];
                s_x[3 * th + i] = a.rh[((size_t)c * a.ntheta + th) * 3 + i];
            }
        }
        __syncthreads();
        if (!act) continue;
        const cplx xJ = c2(a.X[(int64_t)c * a.ldx + n]), xM = c2(a.X[(int64_t)c * a.ldx + a.N + n]);
        for (int p = 0; p < Nq; p++) {
            const double u[3] = {rp[p][0] - vF[0], rp[p][1] - vF[1], rp[p][2] - vF[2]};
            cplx ag[3] = {{0, 0}, {0, 0}, {0, 0}}, aF[3] = {{0, 0}, {0, 0}, {0, 0}}, aa = {0, 0};
            for (int th = 0; th < a.ntheta; th++) {
                const double* r = s_r + 3 * th;
                const double rd = r[0] * rp[p][0] + r[1] * rp[p][1] + r[2] * rp[p][2];
                double sn, cs;
                sincos(a.kr * rd, &sn, &cs);
                const double ea = a.ki != 0.0 ? exp(a.ki * rd) : 1.0;
                const cplx ph = {ea * cs, -ea * sn};  // exp(-ik rhat.r)
                cplx Y[3];
                for (int i = 0; i < 3; i++)
                    Y[i] = cadd(cscale(cmul(xJ, c2(s_h[3 * th + i])), a.eta), cmul(xM, c2(s_x[3 * th + i])));
                const cplx uY = cadd(cadd(cscale(Y[0], u[0]), cscale(Y[1], u[1])), cscale(Y[2], u[2]));
                const cplx pY = cmul(ph, uY);
                const cplx mp = cmul(mik, pY);
                for (int i = 0; i < 3; i++) {
                    const cplx py = cmul(ph, Y[i]);
                    ag[i] = cadd(ag[i], cadd(py, cscale(mp, r[i])));
                    aF[i] = cadd(aF[i], py);
                }
                aa = cadd(aa, pY);
            }
            const double w = a.q.w[p];
            for (int i = 0; i < 3; i++) {
                grp[p][i] += al * w * cmul(pk, ag[i]).re;
                gF[i] -= al * w * cmul(pk, aF[i]).re;
            }
            gal += w * cmul(pk, aa).re;
        }
    }
    if (!act) return;
    double gv[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int p = 0; p < Nq; p++) {
        const double l1 = a.q.l1[p], l2 = a.q.l2[p], l0 = 1.0 - l1 - l2;
        for (int c = 0; c < 3; c++) {
            gv[c] += l0 * grp[p][c];
            gv[3 + c] += l1 * grp[p][c];
            gv[6 + c] += l2 * grp[p][c];
        }
    }
    for (int c = 0; c < 3; c++) gv[3 * jf + c] += gF[c];
    alpha_to_vertices(v, sign, jf, gal, gv);
    for (int j = 0; j < 9; j++) a.ghalf[9 * (size_t)hn + j] = gv[j];
}

// S = (Lam Xd^T + Xd Lam^T) / 2 -> the four N x N weight matrices
__global__ void weights_kernel(const double2* __restrict__ S, int N, double eta_e, double eta_i,
                               double2* __restrict__ WLe, double2* __restrict__ WLi, double2* __restrict__ WK,
                               double2* __restrict__ Weta) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)N * N) return;
    const int m = (int)(i / N), n = (int)(i % N);
    const int64_t ld = 2 * (int64_t)N;
    const double2 s11 = S[m * ld + n], s22 = S[(N + m) * ld + N + n], s12 = S[m * ld + N + n],
                  s21 = S[(N + m) * ld + n];
    WLe[i] = make_double2(eta_e * s11.x - s22.x / eta_e, eta_e * s11.y - s22.y / eta_e);
    WLi[i] = make_double2(eta_i * s11.x - s22.x / eta_i, eta_i * s11.y - s22.y / eta_i);
    WK[i] = make_double2(s12.x + s21.x, s12.y + s21.y);
    const double ie2 = 1.0 / (eta_i * eta_i);
    Weta[i] = make_double2(s11.x + s22.x * ie2, s11.y + s22.y * ie2);
}

// Y[i][c] = s(i) X[c][i]: column-major n x nc -> row-major n x nc, rows >= flip negated
__global__ void transpose_flip_kernel(const double2* __restrict__ X, int64_t ldx, int n, int nc, int flip_from,
                                      double2* __restrict__ Y) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)n * nc) return;
    const int r = (int)(i / nc), c = (int)(i % nc);
    double2 v = X[(int64_t)c * ldx + r];
    if (r >= flip_from) v = make_double2(-v.x, -v.y);
    Y[i] = v;
}

struct DevBuf {
    void* p = nullptr;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    int alloc(bem_ctx* ctx, size_t bytes) {
        if (cudaMalloc(&p, bytes) != cudaSuccess) {
            cudaGetLastError();
            p = nullptr;
            return fail(ctx, BEM_ERR_OOM, "gradient buffer of %zu bytes", bytes);
        }
        return BEM_OK;
    }
};

unsigned nblocks(int64_t n, int b) { return (unsigned)((n + b - 1) / b); }

}  // namespace

int adjoint_geometry(bem_ctx* ctx, const bem_geom* g, std::complex<double> kext, std::complex<double> kint,
                     double eta_e, double eta_i, unsigned flags, const void* X, const void* Lam, int ncols,
                     const double* RT_dev, int n_orient, const void* hp_dev, const void* rh_dev, int ntheta,
                     double* grad_v, double* dpsi_dk, double* dpsi_deta) {
    const int N = g->N, n = 2 * N, nt = g->nt, Nq = g->Nq, nv = g->nv;
    cudaStream_t st = ctx->stream;
    // per-triangle halves and per-half (triangle, local free vertex)
    std::vector<int> hinfo((size_t)nt * 9, -1), htri(2 * (size_t)N), hjf(2 * (size_t)N);
    std::vector<int> cnt(nt, 0);
    const HostMesh& M = g->mesh;
    const HostRWG& r = g->rwg;
    for (int h = 0; h < 2; h++)
        for (int m = 0; m < N; m++) {
            const int t = h == 0 ? r.tri_p[m] : r.tri_m[m];
            const int vf = h == 0 ? r.vfree_p[m] : r.vfree_m[m];
            int jf = -1;
            for (int j = 0; j < 3; j++)
                if (M.tris[3 * t + j] == vf) jf = j;
            if (jf < 0 || cnt[t] >= 3) return fail(ctx, BEM_ERR_INVALID, "RWG %d: free vertex not on triangle %d", m, t);
            const int k = cnt[t]++;
            hinfo[((size_t)t * 3 + k) * 3] = m;
            hinfo[((size_t)t * 3 + k) * 3 + 1] = h == 0 ? 1 : -1;
            hinfo[((size_t)t * 3 + k) * 3 + 2] = jf;
            htri[(size_t)h * N + m] = t;
            hjf[(size_t)h * N + m] = jf;
        }
    TriQ tq;
    tq.n = g->quad.n;
    for (int i = 0; i < 25; i++) tq.l1[i] = g->quad.l1[i], tq.l2[i] = g->quad.l2[i], tq.w[i] = g->quad.w[i];
    const size_t NN = (size_t)N * N;
    DevBuf dS, dW, dT, dInfo, dOut;
    BEM_TRY(dS.alloc(ctx, (size_t)n * n * sizeof(double2)));
    BEM_TRY(dW.alloc(ctx, 4 * NN * sizeof(double2)));
    BEM_TRY(dT.alloc(ctx, 2 * (size_t)n * ncols * sizeof(double2)));
    BEM_TRY(dInfo.alloc(ctx, (hinfo.size() + 4 * (size_t)N) * sizeof(int)));
    const size_t out_dbl = 2 * (size_t)nt * 9 + 10 * (size_t)nt + 2 * (size_t)n * 9;
    BEM_TRY(dOut.alloc(ctx, out_dbl * sizeof(double)));
    int* d_hinfo = (int*)dInfo.p;
    int* d_htri = d_hinfo + hinfo.size();
    int* d_hjf = d_htri + 2 * N;
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(d_hinfo, hinfo.data(), hinfo.size() * 4, cudaMemcpyHostToDevice, st));
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(d_htri, htri.data(), htri.size() * 4, cudaMemcpyHostToDevice, st));
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(d_hjf, hjf.data(), hjf.size() * 4, cudaMemcpyHostToDevice, st));
    // S = (Lam Xd^T + Xd Lam^T) / 2, Xd = D X
    double2* LT = (double2*)dT.p;
    double2* XT = LT + (size_t)n * ncols;
    const int64_t nx = (int64_t)n * ncols;
    transpose_flip_kernel<<<nblocks(nx, 256), 256, 0, st>>>((const double2*)Lam, n, n, ncols, n, LT);
    BEM_LAUNCHED(ctx);
    transpose_flip_kernel<<<nblocks(nx, 256), 256, 0, st>>>((const double2*)X, n, n, ncols, N, XT);
    BEM_LAUNCHED(ctx);
    double2* S = (double2*)dS.p;
    BEM_TRY_CUDA(ctx, cudaMemsetAsync(S, 0, (size_t)n * n * sizeof(double2), st));
    BEM_TRY(cgemm<double>(ctx, n, n, ncols, LT, ncols, XT, ncols, true, S, n, false, make_double2(0.5, 0),
                          make_double2(1, 0)));
    BEM_TRY(cgemm<double>(ctx, n, n, ncols, XT, ncols, LT, ncols, true, S, n, false, make_double2(0.5, 0),
                          make_double2(1, 0)));
    double2* W = (double2*)dW.p;
    weights_kernel<<<nblocks((int64_t)NN, 256), 256, 0, st>>>(S, N, eta_e, eta_i, W, W + NN, W + 2 * NN, W + 3 * NN);
    BEM_LAUNCHED(ctx);
    GradWeights gw{W, W + NN, W + 2 * NN, W + 3 * NN, N};
    double* o_pair = (double*)dOut.p;
    double* o_self = o_pair + (size_t)nt * 9;
    double* o_skp = o_self + (size_t)nt * 9;
    double* o_sep = o_skp + 2 * (size_t)nt;
    double* o_sks = o_sep + 2 * (size_t)nt;
    double* o_ses = o_sks + 4 * (size_t)nt;
    double* o_rhs = o_ses + 2 * (size_t)nt;
    double* o_ff = o_rhs + (size_t)n * 9;
    const Medium ke{kext.real(), kext.imag()}, ki{kint.real(), kint.imag()};
    PairArgs pa{g->sing.tv, d_hinfo, nt, Nq, tq, ke, ki, gw, o_pair, o_skp, o_sep};
    grad_pair_kernel<<<nt, 128, 0, st>>>(pa);
    BEM_LAUNCHED(ctx);
    SelfArgs sa{g->sing.tv, d_hinfo, nt, Nq, tq, ke, ki, flags, gw, o_self, o_sks, o_ses};
    grad_self_kernel<<<nblocks(nt, 64), 64, 0, st>>>(sa);
    BEM_LAUNCHED(ctx);
    HalfArgs ha{g->sing.tv, d_htri, d_hjf, N, Nq, tq, kext.real(), kext.imag(), eta_e, RT_dev, n_orient,
                (const double2*)Lam, n, o_rhs};
    grad_rhs_kernel<<<nblocks(n, 64), 64, 0, st>>>(ha);
    BEM_LAUNCHED(ctx);
    FFArgs2 fa{g->sing.tv, d_htri, d_hjf, N, Nq, tq, kext.real(), kext.imag(), eta_e, RT_dev, ntheta, ncols,
               (const double2*)hp_dev, (const double2*)rh_dev, (const double2*)X, n, o_ff};
    const size_t smem = (size_t)((3 * ntheta + 1) & ~1) * 8 + (size_t)ntheta * 6 * 16;
    if (smem > 200 * 1024) return fail(ctx, BEM_ERR_INVALID, "ntheta %d too large for the far-field gradient", ntheta);
    BEM_TRY_CUDA(ctx, cudaFuncSetAttribute(grad_ff_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    grad_ff_kernel<<<nblocks(n, 32), 32, smem, st>>>(fa);
    BEM_LAUNCHED(ctx);
    std::vector<double> out(out_dbl);
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(out.data(), dOut.p, out_dbl * 8, cudaMemcpyDeviceToHost, st));
    BEM_TRY_CUDA(ctx, cudaStreamSynchronize(st));
    const double* h_pair = out.data();
    const double* h_self = h_pair + (size_t)nt * 9;
    const double* h_skp = h_self + (size_t)nt * 9;
    const double* h_sep = h_skp + 2 * (size_t)nt;
    const double* h_sks = h_sep + 2 * (size_t)nt;
    const double* h_ses = h_sks + 4 * (size_t)nt;
    const double* h_rhs = h_ses + 2 * (size_t)nt;
    const double* h_ff = h_rhs + (size_t)n * 9;
    if (grad_v) {
        std::fill(grad_v, grad_v + 3 * (size_t)nv, 0.0);
        for (int t = 0; t < nt; t++)
            for (int j = 0; j < 3; j++)
                for (int c = 0; c < 3; c++)
                    grad_v[3 * (size_t)M.tris[3 * t + j] + c] -= h_pair[9 * t + 3 * j + c] + h_self[9 * t + 3 * j + c];
        for (int hn = 0; hn < n; hn++) {
            const int t = htri[hn];
            for (int j = 0; j < 3; j++)
                for (int c = 0; c < 3; c++)
                    grad_v[3 * (size_t)M.tris[3 * t + j] + c] +=
                        h_rhs[9 * (size_t)hn + 3 * j + c] + h_ff[9 * (size_t)hn + 3 * j + c];
        }
    }
    // pair terms are holomorphic in k: d/dIm k = i d/dRe k
    double skr[2] = {0, 0}, ski[2] = {0, 0}, se[2] = {0, 0};
    for (int t = 0; t < nt; t++) {
        skr[0] += h_skp[2 * t] + h_sks[4 * t], skr[1] += h_skp[2 * t + 1] + h_sks[4 * t + 1];
        ski[0] += -h_skp[2 * t + 1] + h_sks[4 * t + 2], ski[1] += h_skp[2 * t] + h_sks[4 * t + 3];
        se[0] += h_sep[2 * t] + h_ses[2 * t], se[1] += h_sep[2 * t + 1] + h_ses[2 * t + 1];
    }
    if (dpsi_dk) dpsi_dk[0] = skr[0], dpsi_dk[1] = skr[1], dpsi_dk[2] = ski[0], dpsi_dk[3] = ski[1];
    if (dpsi_deta) dpsi_deta[0] = se[0], dpsi_deta[1] = se[1];
    return BEM_OK;
}

}  // namespace bem
