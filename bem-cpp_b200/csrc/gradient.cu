// Adjoint gradient of an orientation-averaged M11 misfit with respect to the
// relative refractive index m = m_re + i m_im.
//
//   loss = sum_t wt_t (M11(theta_t) - target_t)^2
//
// One FP64 forward solve X = Z^-1 B, the far field F of every column, the
// adjoint right-hand sides g_c = dloss/dx_c (an adjoint far-field kernel),
// one adjoint solve with the same factors (the PMCHWT Z satisfies
// Z^T = D Z D, D = diag(I, -I), so Z^-T g = D Z^-1 D g), and the operator
// derivatives dZ/dm_re, dZ/dm_im from central differences of the assembled Z
// in m (the exterior blocks cancel exactly):
//   dloss/dp = -Re sum_c lambda_c^T (dZ/dp) x_c,   lambda = Z^-T g.
// The reference has no gradient code; this follows its forward path (the
// dense branch of main.cpp:660-854) and is checked against central
// differences of that forward path.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>

#include "bem_internal.h"
#include "lu_internal.h"

namespace bem {

constexpr double INV4PI_G = 0.07957747154594767;  // 1 / (4 pi)

struct AdjFFArgs {
    DevHalf h;
    int N, Nq, ntheta, ncols;
    double kr, ki, eta;
    const double* RT;    // n_orient * 9
    const double2* hp;   // [c][theta][3]: the transverse adjoint weight h
    const double2* rh;   // [c][theta][3]: rhat x h
    double2* G;          // column-major n x ncols
    int64_t ldg;
};

// Thread per RWG n, grid (RWG blocks, columns): sums over the directions of
// the column's orientation and the 2 Nq points of n.
__global__ void __launch_bounds__(128) farfield_adjoint_kernel(AdjFFArgs a) {
    extern __shared__ __align__(16) double sm[];
    double* s_r = sm;                                        // ntheta * 3 (padded to 16 bytes)
    double2* s_h = (double2*)(sm + ((3 * a.ntheta + 1) & ~1));  // ntheta * 3
    double2* s_x = s_h + 3 * a.ntheta;                       // ntheta * 3
    const int c = blockIdx.y, o = c / 2;
    for (int t = threadIdx.x; t < a.ntheta; t += blockDim.x) {
        const double th = a.ntheta > 1 ? M_PI * t / (a.ntheta - 1) : 0.0;
        double st, ct;
        sincos(th, &st, &ct);
        const double* R = a.RT + 9 * o;
        for (int i = 0; i < 3; i++) s_r[3 * t + i] = R[3 * i] * st + R[3 * i + 2] * ct;
        for (int i = 0; i < 3; i++) {
            s_h[3 * t + i] = a.hp[((size_t)c * a.ntheta + t) * 3 + i];
            s_x[3 * t + i] = a.rh[((size_t)c * a.ntheta + t) * 3 + i];
        }
    }
    __syncthreads();
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= a.N) return;
    double gj[2] = {0, 0}, gm[2] = {0, 0};
    for (int hh = 0; hh < 2; hh++)
        for (int q = 0; q < a.Nq; q++) {
            const size_t p = ((size_t)hh * a.N + n) * a.Nq + q;
            const double px = a.h.px[p], py = a.h.py[p], pz = a.h.pz[p], w = a.h.jw[p];
            const double fx = a.h.fx[p] * w, fy = a.h.fy[p] * w, fz = a.h.fz[p] * w;
            for (int t = 0; t < a.ntheta; t++) {
                const double rd = s_r[3 * t] * px + s_r[3 * t + 1] * py + s_r[3 * t + 2] * pz;
                double sn, cs;
                sincos(a.kr * rd, &sn, &cs);
                const double ea = a.ki != 0.0 ? exp(a.ki * rd) : 1.0;
                const double er = cs * ea, ei = -sn * ea;  // exp(-i k rhat.r)
                const double2* hv = s_h + 3 * t;
                const double2* xv = s_x + 3 * t;
                const double dr = fx * hv[0].x + fy * hv[1].x + fz * hv[2].x;
                const double di = fx * hv[0].y + fy * hv[1].y + fz * hv[2].y;
                const double mr = fx * xv[0].x + fy * xv[1].x + fz * xv[2].x;
                const double mi = fx * xv[0].y + fy * xv[1].y + fz * xv[2].y;
                gj[0] += er * dr - ei * di;
                gj[1] += er * di + ei * dr;
                gm[0] += er * mr - ei * mi;
                gm[1] += er * mi + ei * mr;
            }
        }
    // -ik/(4 pi) = (k_im - i k_re)/(4 pi); the J part also carries eta
    const double pr = a.ki * INV4PI_G, pi_ = -a.kr * INV4PI_G;
    double2 vj, vm;
    vj.x = a.eta * (pr * gj[0] - pi_ * gj[1]);
    vj.y = a.eta * (pr * gj[1] + pi_ * gj[0]);
    vm.x = pr * gm[0] - pi_ * gm[1];
    vm.y = pr * gm[1] + pi_ * gm[0];
    a.G[(int64_t)c * a.ldg + n] = vj;
    a.G[(int64_t)c * a.ldg + a.N + n] = vm;
}

// partial[b] = sum over this block's entries of L[i] R[i] (complex, no conjugate)
__global__ void cdot_kernel(const double2* __restrict__ L, const double2* __restrict__ R, int64_t count,
                            double2* __restrict__ partial) {
    __shared__ double sr[256], si[256];
    double ar = 0, ai = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x) {
        const double2 l = L[i], r = R[i];
        ar += l.x * r.x - l.y * r.y;
        ai += l.x * r.y + l.y * r.x;
    }
    sr[threadIdx.x] = ar;
    si[threadIdx.x] = ai;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            sr[threadIdx.x] += sr[threadIdx.x + o];
            si[threadIdx.x] += si[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = make_double2(sr[0], si[0]);
}

// rows [r0, n) of every column negated (D = diag(I, -I) applied to a block)
__global__ void flip_rows_kernel(double2* __restrict__ X, int64_t ldx, int r0, int n, int ncols) {
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int m = n - r0;
    if (t >= (int64_t)m * ncols) return;
    const int r = r0 + (int)(t % m), c = (int)(t / m);
    double2 v = X[(int64_t)c * ldx + r];
    X[(int64_t)c * ldx + r] = make_double2(-v.x, -v.y);
}

// Y = A - B elementwise, scaled by s
__global__ void diff_scale_kernel(const double2* __restrict__ A, const double2* __restrict__ B, double s,
                                  double2* __restrict__ Y, int64_t count) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    Y[i] = make_double2((A[i].x - B[i].x) * s, (A[i].y - B[i].y) * s);
}

namespace {
struct DevMem {
    void* p = nullptr;
    ~DevMem() {
        if (p) cudaFree(p);
    }
};
unsigned blocks_for(int64_t n) { return (unsigned)std::min<int64_t>((n + 255) / 256, 1 << 30); }
}  // namespace

}  // namespace bem

using namespace bem;

// Forward solve, adjoint solve, then the requested gradients: with respect to
// (Re m, Im m) (grad_m, 2 values) and/or the vertex coordinates (grad_v, 3 nv
// values).  The vertex derivatives use, per coordinate, the operator, the
// right-hand sides and the far field (at fixed coefficients) assembled on
// the geometry moved by +-h:
//   dloss/dv = Re sum_c lambda_c^T (dB_c/dv - dZ/dv x_c) + dloss/dv|_x
static int adjoint_core(bem_ctx* ctx, const bem_problem* p, const double* target, const double* wt,
                        double* loss_out, double* grad_out, double* grad_v, double* mueller_out) {
    if (!ctx || !p || !target || !loss_out || (!grad_out && !grad_v)) return BEM_ERR_INVALID;
    if (!(p->ka > 0) || p->ntheta < 2) return fail(ctx, BEM_ERR_INVALID, "ka must be > 0, ntheta >= 2");
    BEM_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    const std::complex<double> m(p->m_re, p->m_im), kext(p->ka, 0.0);
    const double eta_e = 1.0;
    bem_geom* g = nullptr;
    int N = 0;
    BEM_TRY(bem_geom_create(ctx, p->verts, p->nv, p->tris, p->nt, p->quad_order, &g, &N));
    struct GeomGuard {
        bem_geom* g;
        ~GeomGuard() { bem_geom_free(g); }
    } gg{g};
    const int n = 2 * N;
    std::vector<double> RT, w;
    if (p->single) {
        RT = {1, 0, 0, 0, 1, 0, 0, 0, 1};
        w = {1.0};
    } else {
        orientations(p->n_alpha, p->n_beta, p->n_gamma, p->beta_sym < 1 ? 1 : p->beta_sym,
                     p->gamma_sym < 1 ? 1 : p->gamma_sym, p->gamma_mirror != 0, true, RT, w);
    }
    const int no = (int)w.size(), nc = 2 * no, nt = p->ntheta;
    const size_t zb = (size_t)n * n * 16, xb = (size_t)n * nc * 16;
    const bool fd = ctx->grad_method == 1;  // derivatives of reassembled operators (else the contraction kernels)
    DevMem dZ, dZp, dX, dB, dL, dY;
    if (cudaMalloc(&dZ.p, zb) != cudaSuccess || (fd && cudaMalloc(&dZp.p, zb) != cudaSuccess) ||
        cudaMalloc(&dX.p, xb) != cudaSuccess || cudaMalloc(&dB.p, xb) != cudaSuccess ||
        cudaMalloc(&dL.p, xb) != cudaSuccess || cudaMalloc(&dY.p, xb) != cudaSuccess) {
        cudaGetLastError();
        return fail(ctx, BEM_ERR_OOM, "gradient buffers for n=%d, %d columns", n, nc);
    }
    auto assemble_m = [&](std::complex<double> mm, void* Zout) {
        const std::complex<double> ki = kext * mm;
        return assemble_dev(ctx, g, kext.real(), kext.imag(), ki.real(), ki.imag(), eta_e, 1.0 / std::abs(mm),
                            p->asm_flags, 2, Zout, n, nullptr, nullptr);
    };
    // forward solve (FP64)
    BEM_TRY(assemble_m(m, dZ.p));
    BEM_TRY(rhs_dev(ctx, g, kext.real(), kext.imag(), eta_e, RT.data(), nullptr, nullptr, no, dB.p, n));
    // the vertex derivatives reassemble only the tiles around a moved vertex
    // into a copy of the unperturbed operator
    DevMem dZbase;
    if (grad_v && fd) {
        if (cudaMalloc(&dZbase.p, zb) != cudaSuccess) {
            cudaGetLastError();
            return fail(ctx, BEM_ERR_OOM, "gradient buffers for n=%d", n);
        }
        BEM_TRY_CUDA(ctx, cudaMemcpyAsync(dZbase.p, dZ.p, zb, cudaMemcpyDeviceToDevice, ctx->stream));
    }
    bem_lu* lu = nullptr;
    int info = 0;
    BEM_TRY(bem_lu_factor_dev(ctx, dZ.p, n, n, BEM_PREC_FP64, &lu, &info));
    struct LuGuard {
        bem_lu* lu;
        ~LuGuard() { bem_lu_free(lu); }
    } lg{lu};
    if (info > 0) return fail(ctx, BEM_ERR_SINGULAR, "zero pivot at %d", info);
    BEM_TRY(bem_lu_solve_dev(ctx, lu, dB.p, n, dX.p, n, nc, 0.0, 0, nullptr));
    // far field of every column and the averaged Mueller matrix
    std::vector<double> M(16 * (size_t)nt), Fv((size_t)nc * nt * 3 * 2);
    BEM_TRY(mueller_dev(ctx, g, dX.p, n, RT.data(), w.data(), no, kext.real(), kext.imag(), eta_e, nt,
                        p->gamma_mirror, M.data(), nullptr, Fv.data()));
    auto misfit = [&](const double* MM) {
        double l = 0.0;
        for (int t = 0; t < nt; t++) {
            const double wtt = wt ? wt[t] : 1.0, r = MM[t] - target[t];
            l += wtt * r * r;
        }
        return l;
    };
    const double loss = misfit(M.data());
    std::vector<double> coef(nt);
    for (int t = 0; t < nt; t++) coef[t] = 2.0 * (wt ? wt[t] : 1.0) * (M[t] - target[t]);
    // adjoint weights: h_c(theta) = coef w_o sum_{e in (e_par, e_perp)} conj(F.e) e, and rhat x h
    std::vector<double> hp((size_t)nc * nt * 3 * 2), rh((size_t)nc * nt * 3 * 2);
    for (int c = 0; c < nc; c++) {
        const int o = c / 2;
        const double* R = RT.data() + 9 * o;
        for (int t = 0; t < nt; t++) {
            const double th = M_PI * t / (nt - 1), st = std::sin(th), ct = std::cos(th);
            double r[3], ep[3], ee[3];
            for (int i = 0; i < 3; i++) {
                r[i] = R[3 * i] * st + R[3 * i + 2] * ct;
                ep[i] = R[3 * i] * ct - R[3 * i + 2] * st;
                ee[i] = R[3 * i + 1];
            }
            const double* F = Fv.data() + ((size_t)c * nt + t) * 6;
            std::complex<double> Fc[3] = {{F[0], F[1]}, {F[2], F[3]}, {F[4], F[5]}};
            std::complex<double> a = std::conj(Fc[0] * ep[0] + Fc[1] * ep[1] + Fc[2] * ep[2]);
            std::complex<double> b = std::conj(Fc[0] * ee[0] + Fc[1] * ee[1] + Fc[2] * ee[2]);
            const double s = coef[t] * w[o];
            std::complex<double> h[3];
            for (int i = 0; i < 3; i++) h[i] = s * (a * ep[i] + b * ee[i]);
            std::complex<double> x[3] = {r[1] * h[2] - r[2] * h[1], r[2] * h[0] - r[0] * h[2],
                                         r[0] * h[1] - r[1] * h[0]};
            double* hq = hp.data() + ((size_t)c * nt + t) * 6;
            double* xq = rh.data() + ((size_t)c * nt + t) * 6;
            for (int i = 0; i < 3; i++) {
                hq[2 * i] = h[i].real(), hq[2 * i + 1] = h[i].imag();
                xq[2 * i] = x[i].real(), xq[2 * i + 1] = x[i].imag();
            }
        }
    }
    DevMem dH, dRh, dRT, dPart;
    const size_t hb = hp.size() * 8;
    if (cudaMalloc(&dH.p, hb) != cudaSuccess || cudaMalloc(&dRh.p, hb) != cudaSuccess ||
        cudaMalloc(&dRT.p, RT.size() * 8) != cudaSuccess || cudaMalloc(&dPart.p, 1024 * 16) != cudaSuccess) {
        cudaGetLastError();
        return fail(ctx, BEM_ERR_OOM, "gradient weights");
    }
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(dH.p, hp.data(), hb, cudaMemcpyHostToDevice, ctx->stream));
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(dRh.p, rh.data(), hb, cudaMemcpyHostToDevice, ctx->stream));
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(dRT.p, RT.data(), RT.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
    AdjFFArgs aa{};
    aa.h = g->half;
    aa.N = N;
    aa.Nq = g->Nq;
    aa.ntheta = nt;
    aa.ncols = nc;
    aa.kr = kext.real();
    aa.ki = kext.imag();
    aa.eta = eta_e;
    aa.RT = (const double*)dRT.p;
    aa.hp = (const double2*)dH.p;
    aa.rh = (const double2*)dRh.p;
    aa.G = (double2*)dY.p;  // g
    aa.ldg = n;
    const size_t smem = (size_t)((3 * nt + 1) & ~1) * 8 + (size_t)nt * 6 * 16;
    if (smem > 200 * 1024) return fail(ctx, BEM_ERR_INVALID, "ntheta %d too large for the adjoint far field", nt);
    BEM_TRY_CUDA(ctx, cudaFuncSetAttribute(farfield_adjoint_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem));
    farfield_adjoint_kernel<<<dim3((N + 127) / 128, nc), 128, smem, ctx->stream>>>(aa);
    BEM_LAUNCHED(ctx);
    // lambda = D Z^-1 D g
    const int64_t half = (int64_t)(n - N) * nc;
    flip_rows_kernel<<<blocks_for(half), 256, 0, ctx->stream>>>((double2*)dY.p, n, N, n, nc);
    BEM_LAUNCHED(ctx);
    BEM_TRY(bem_lu_solve_dev(ctx, lu, dY.p, n, dL.p, n, nc, 0.0, 0, nullptr));
    flip_rows_kernel<<<blocks_for(half), 256, 0, ctx->stream>>>((double2*)dL.p, n, N, n, nc);
    BEM_LAUNCHED(ctx);
    // sum over all entries of lambda . Y (complex, no conjugate)
    std::vector<double> part(2048);
    auto dot_lambda = [&](const void* Y, double* re) {
        cdot_kernel<<<1024, 256, 0, ctx->stream>>>((const double2*)dL.p, (const double2*)Y, (int64_t)n * nc,
                                                  (double2*)dPart.p);
        BEM_LAUNCHED(ctx);
        BEM_TRY_CUDA(ctx, cudaMemcpyAsync(part.data(), dPart.p, 1024 * 16, cudaMemcpyDeviceToHost, ctx->stream));
        BEM_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        double tr = 0;
        for (int i = 0; i < 1024; i++) tr += part[2 * i];
        *re = tr;
        return (int)BEM_OK;
    };
    if (!fd) {
        // the contraction kernels (grad_geom.cu): vertex gradient, and the
        // interior wavenumber / impedance contractions for m
        const double am = std::abs(m), am3 = am * am * am;
        double dk[4] = {0, 0, 0, 0}, deta[2] = {0, 0};
        BEM_TRY(adjoint_geometry(ctx, g, kext, kext * m, eta_e, 1.0 / am, p->asm_flags, dX.p, dL.p, nc,
                                 (const double*)dRT.p, no, dH.p, dRh.p, nt, grad_v, dk, deta));
        if (grad_out) {
            // k_i = k_e m with k_e real: d/dRe m = k_e d/dRe k_i, d/dIm m = k_e d/dIm k_i;
            // eta_i = 1/|m|
            grad_out[0] = -(kext.real() * dk[0] + (-m.real() / am3) * deta[0]);
            grad_out[1] = -(kext.real() * dk[2] + (-m.imag() / am3) * deta[0]);
        }
        *loss_out = loss;
        if (mueller_out) std::memcpy(mueller_out, M.data(), M.size() * 8);
        return BEM_OK;
    }
    // dZ/dp by central differences in m, contracted with lambda and x
    const double delta = 1e-5;
    for (int comp = 0; grad_out && comp < 2; comp++) {
        const std::complex<double> dm = comp == 0 ? std::complex<double>(delta, 0) : std::complex<double>(0, delta);
        BEM_TRY(assemble_m(m + dm, dZ.p));
        BEM_TRY(assemble_m(m - dm, dZp.p));
        const int64_t nn = (int64_t)n * n;
        diff_scale_kernel<<<blocks_for(nn), 256, 0, ctx->stream>>>((const double2*)dZ.p, (const double2*)dZp.p,
                                                                  0.5 / delta, (double2*)dZ.p, nn);
        BEM_LAUNCHED(ctx);
        // Y = -dZ X, then t = sum lambda . Y = -sum lambda^T dZ x
        BEM_TRY_CUDA(ctx, cudaMemsetAsync(dY.p, 0, xb, ctx->stream));
        BEM_TRY(cgemm<double>(ctx, n, nc, n, (const double2*)dZ.p, n, (const double2*)dX.p, n, true, (double2*)dY.p,
                              n, true, make_double2(-1, 0), make_double2(1, 0)));
        double tr = 0;
        BEM_TRY(dot_lambda(dY.p, &tr));
        grad_out[comp] = tr;  // Re(-sum lambda^T dZ x)
    }
    if (grad_v) {
        // per vertex coordinate: Z, B and the far field on the geometry moved by +-h
        const double h = 1e-6;
        std::vector<double> vp(p->verts, p->verts + 3 * (size_t)p->nv);
        std::vector<double> Mp(16 * (size_t)nt), Mm(16 * (size_t)nt);
        DevMem dBm;
        if (cudaMalloc(&dBm.p, xb) != cudaSuccess) {
            cudaGetLastError();
            return fail(ctx, BEM_ERR_OOM, "gradient buffers");
        }
        const std::complex<double> ki = kext * m;
        // RWGs around each vertex (the RWGs with a triangle on it): the
        // entries the vertex moves; assembly recomputes only their tiles
        std::vector<std::vector<int>> vrwg(p->nv);
        for (int mm = 0; mm < N; mm++)
            for (int tri : {g->rwg.tri_p[mm], g->rwg.tri_m[mm]})
                for (int k = 0; k < 3; k++) {
                    auto& vr = vrwg[p->tris[3 * tri + k]];
                    if (vr.empty() || vr.back() != mm) vr.push_back(mm);
                }
        DevMem dMask;
        if (cudaMalloc(&dMask.p, N) != cudaSuccess) {
            cudaGetLastError();
            return fail(ctx, BEM_ERR_OOM, "gradient buffers");
        }
        std::vector<unsigned char> mask(N);
        // one working geometry, moved in place per evaluation (same topology,
        // tiles and device arrays as a geometry created from the moved mesh)
        struct GeomGuard {
            bem_geom* g = nullptr;
            ~GeomGuard() {
                if (g) bem_geom_free(g);
            }
        } gw;
        {
            int Nw = 0;
            BEM_TRY(bem_geom_create(ctx, vp.data(), p->nv, p->tris, p->nt, p->quad_order, &gw.g, &Nw));
            if (Nw != N) return fail(ctx, BEM_ERR_INVALID, "working geometry has %d RWGs, not %d", Nw, N);
        }
        for (int iv = 0; iv < p->nv; iv++) {
            std::fill(mask.begin(), mask.end(), 0);
            for (int mm : vrwg[iv]) mask[mm] = 1;
            BEM_TRY_CUDA(ctx, cudaMemcpyAsync(dMask.p, mask.data(), N, cudaMemcpyHostToDevice, ctx->stream));
            for (int comp = 0; comp < 3; comp++) {
                const double v0 = vp[3 * iv + comp];
                double lpm[2] = {0, 0};
                void* Zs[2] = {dZ.p, dZp.p};
                void* Bs[2] = {dB.p, dBm.p};
                double* Ms[2] = {Mp.data(), Mm.data()};
                for (int sgn = 0; sgn < 2; sgn++) {
                    vp[3 * iv + comp] = v0 + (sgn == 0 ? h : -h);
                    bem_geom* gs = gw.g;
                    int st = geom_set_vertices(ctx, gs, vp.data());
                    if (st == BEM_OK && cudaMemcpyAsync(Zs[sgn], dZbase.p, zb, cudaMemcpyDeviceToDevice,
                                                        ctx->stream) != cudaSuccess)
                        st = fail(ctx, BEM_ERR_CUDA, "operator copy");
                    if (st == BEM_OK)
                        st = assemble_dev(ctx, gs, kext.real(), kext.imag(), ki.real(), ki.imag(), eta_e,
                                          1.0 / std::abs(m), p->asm_flags, 2, Zs[sgn], n, nullptr, nullptr,
                                          (const unsigned char*)dMask.p);
                    if (st == BEM_OK)
                        st = rhs_dev(ctx, gs, kext.real(), kext.imag(), eta_e, RT.data(), nullptr, nullptr, no,
                                     Bs[sgn], n);
                    if (st == BEM_OK)
                        st = mueller_dev(ctx, gs, dX.p, n, RT.data(), w.data(), no, kext.real(), kext.imag(), eta_e,
                                         nt, p->gamma_mirror, Ms[sgn], nullptr);
                    if (st != BEM_OK) {
                        vp[3 * iv + comp] = v0;
                        return st;
                    }
                    lpm[sgn] = misfit(Ms[sgn]);
                }
                vp[3 * iv + comp] = v0;
                const double inv2h = 0.5 / h;
                const int64_t nn = (int64_t)n * n, nx = (int64_t)n * nc;
                // -dZ/dv x
                diff_scale_kernel<<<blocks_for(nn), 256, 0, ctx->stream>>>((const double2*)dZ.p, (const double2*)dZp.p,
                                                                          inv2h, (double2*)dZ.p, nn);
                BEM_LAUNCHED(ctx);
                BEM_TRY_CUDA(ctx, cudaMemsetAsync(dY.p, 0, xb, ctx->stream));
                BEM_TRY(cgemm<double>(ctx, n, nc, n, (const double2*)dZ.p, n, (const double2*)dX.p, n, true,
                                      (double2*)dY.p, n, true, make_double2(-1, 0), make_double2(1, 0)));
                double t_z = 0, t_b = 0;
                BEM_TRY(dot_lambda(dY.p, &t_z));
                // dB/dv
                diff_scale_kernel<<<blocks_for(nx), 256, 0, ctx->stream>>>((const double2*)dB.p, (const double2*)dBm.p,
                                                                          inv2h, (double2*)dY.p, nx);
                BEM_LAUNCHED(ctx);
                BEM_TRY(dot_lambda(dY.p, &t_b));
                grad_v[3 * iv + comp] = t_z + t_b + (lpm[0] - lpm[1]) * inv2h;
            }
        }
    }
    *loss_out = loss;
    if (mueller_out) std::memcpy(mueller_out, M.data(), M.size() * 8);
    return BEM_OK;
}

extern "C" int bem_adjoint_grad(bem_ctx* ctx, const bem_problem* p, const double* target, const double* wt,
                                double* loss, double* grad, double* mueller) {
    if (!grad) return BEM_ERR_INVALID;
    return adjoint_core(ctx, p, target, wt, loss, grad, nullptr, mueller);
}

extern "C" int bem_adjoint_grad_vertices(bem_ctx* ctx, const bem_problem* p, const double* target, const double* wt,
                                         double* loss, double* grad_verts, double* mueller) {
    if (!grad_verts) return BEM_ERR_INVALID;
    return adjoint_core(ctx, p, target, wt, loss, nullptr, grad_verts, mueller);
}
