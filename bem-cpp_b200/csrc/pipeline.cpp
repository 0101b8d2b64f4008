// Host-buffer assembly mirrors and the whole dense pipeline (the dense branch
// of main.cpp:660-854) over the device kernels.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "bem_internal.h"

using namespace bem;

namespace {

// Device buffer from the device-memory cache (devmem_alloc): a batch of
// particles of one size allocates its buffers once.
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    int device = -1;
    const void* owner = nullptr;
    bool alloc(const bem_ctx* ctx, size_t b) {
        p = devmem_alloc(ctx->device, b, ctx);
        bytes = b;
        device = ctx->device;
        owner = ctx;
        return p != nullptr;
    }
    void release() {
        if (p) devmem_free(device, p, bytes, owner);
        p = nullptr;
    }
    ~DevBuf() { release(); }
};

double secs(std::chrono::steady_clock::time_point a) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - a).count();
}

}  // namespace

extern "C" {

// assemble_L_K_cuda (assembly.h:11-13): L, K host row-major N x N complex128.
int bem_assemble_L_K(bem_ctx* ctx, const double* verts, int nv, const int* tris, int nt, double k_re,
                     double k_im, int quad_order, double* L, double* K) {
    if (!ctx || !L || !K) return BEM_ERR_INVALID;
    bem_geom* g = nullptr;
    int N = 0;
    BEM_TRY(bem_geom_create(ctx, verts, nv, tris, nt, quad_order, &g, &N));
    size_t bytes = (size_t)N * N * 16;
    DevBuf dL, dK;
    int s = BEM_OK;
    if (!dL.alloc(ctx, bytes) || !dK.alloc(ctx, bytes)) {
        cudaGetLastError();
        s = fail(ctx, BEM_ERR_OOM, "L/K device buffers");
    }
    if (s == BEM_OK) s = assemble_dev(ctx, g, k_re, k_im, 0, 0, 1, 1, 0, 1, nullptr, N, dL.p, dK.p);
    if (s == BEM_OK) s = d2h(ctx, L, dL.p, bytes);
    if (s == BEM_OK) s = d2h(ctx, K, dK.p, bytes);
    bem_geom_free(g);
    return s;
}

// assemble_pmchwt (pmchwt.h:12-18): Z host row-major 2N x 2N; L_ext, K_ext optional.
int bem_assemble_pmchwt(bem_ctx* ctx, const double* verts, int nv, const int* tris, int nt,
                        double kext_re, double kext_im, double kint_re, double kint_im, double eta_ext,
                        double eta_int, int quad_order, double* Z, double* L_ext, double* K_ext) {
    if (!ctx || !Z) return BEM_ERR_INVALID;
    bem_geom* g = nullptr;
    int N = 0;
    BEM_TRY(bem_geom_create(ctx, verts, nv, tris, nt, quad_order, &g, &N));
    size_t zb = (size_t)4 * N * N * 16;
    DevBuf dZ;
    int s = BEM_OK;
    if (!dZ.alloc(ctx, zb)) {
        cudaGetLastError();
        s = fail(ctx, BEM_ERR_OOM, "Z device buffer (%zu bytes)", zb);
    }
    if (s == BEM_OK)
        s = assemble_dev(ctx, g, kext_re, kext_im, kint_re, kint_im, eta_ext, eta_int, 0, 2, dZ.p, 2 * N,
                         nullptr, nullptr);
    if (s == BEM_OK) s = d2h(ctx, Z, dZ.p, zb);
    if (s == BEM_OK && (L_ext || K_ext)) {
        size_t b = (size_t)N * N * 16;
        DevBuf dL, dK;
        if (!dL.alloc(ctx, b) || !dK.alloc(ctx, b)) {
            cudaGetLastError();
            s = fail(ctx, BEM_ERR_OOM, "L/K device buffers");
        }
        if (s == BEM_OK) s = assemble_dev(ctx, g, kext_re, kext_im, 0, 0, 1, 1, 0, 1, nullptr, N, dL.p, dK.p);
        if (s == BEM_OK && L_ext) s = d2h(ctx, L_ext, dL.p, b);
        if (s == BEM_OK && K_ext) s = d2h(ctx, K_ext, dK.p, b);
    }
    bem_geom_free(g);
    return s;
}

// main.cpp:660-854 on the device.
int bem_dense_run(bem_ctx* ctx, const bem_problem* p, bem_result* r) {
    if (!ctx || !p || !r || !r->mueller) return BEM_ERR_INVALID;
    if (!(p->ka > 0) || p->ntheta < 2) return fail(ctx, BEM_ERR_INVALID, "ka must be > 0, ntheta >= 2");
    auto t_all = std::chrono::steady_clock::now();
    BEM_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    std::complex<double> m(p->m_re, p->m_im), kext(p->ka, 0.0), kint = kext * m;
    double eta_e = 1.0, eta_i = 1.0 / std::abs(m);
    bem_geom* g = nullptr;
    int N = 0;
    BEM_TRY(bem_geom_create(ctx, p->verts, p->nv, p->tris, p->nt, p->quad_order, &g, &N));
    const int n = 2 * N;
    // orientations
    std::vector<double> RT, w;
    if (p->single) {
        RT = {1, 0, 0, 0, 1, 0, 0, 0, 1};
        w = {1.0};
    } else {
        orientations(p->n_alpha, p->n_beta, p->n_gamma, p->beta_sym < 1 ? 1 : p->beta_sym,
                     p->gamma_sym < 1 ? 1 : p->gamma_sym, p->gamma_mirror != 0, true, RT, w);
        int tot = (int)w.size(), i0 = 0, i1 = tot;
        if (p->orient_i0 >= 0 && p->orient_i1 > p->orient_i0) {
            i0 = std::min(p->orient_i0, tot);
            i1 = std::min(p->orient_i1, tot);
        }
        RT = std::vector<double>(RT.begin() + 9 * i0, RT.begin() + 9 * i1);
        w = std::vector<double>(w.begin() + i0, w.begin() + i1);
    }
    const int no = (int)w.size();
    const int nt = p->ntheta;
    // orientation batches: the whole set at once, or the reference's check
    // interval for adaptive stopping (main.cpp:478)
    const bool adaptive = p->orient_tol > 0 && !p->single;
    const int batch = adaptive ? std::max(20, no / 20) : no;
    const int nrhs_max = 2 * std::min(batch, no);
    const bool gm = p->solver == BEM_SOLVER_GMRES_AEXT;
    if (p->solver != BEM_SOLVER_LU && !gm) {
        bem_geom_free(g);
        return fail(ctx, BEM_ERR_INVALID, "unknown solver %d", p->solver);
    }
    DevBuf dZ, dB, dX, dMo, dA;
    int s = BEM_OK;
    if (!dZ.alloc(ctx, (size_t)n * n * 16) || !dB.alloc(ctx, (size_t)n * nrhs_max * 16) ||
        !dX.alloc(ctx, (size_t)n * nrhs_max * 16) || !dMo.alloc(ctx, (size_t)std::min(batch, no) * 16 * nt * 8) ||
        (gm && !dA.alloc(ctx, (size_t)n * n * 16))) {
        cudaGetLastError();
        bem_geom_free(g);
        return fail(ctx, BEM_ERR_OOM, "pipeline buffers for n=%d, nrhs=%d", n, nrhs_max);
    }
    auto t0 = std::chrono::steady_clock::now();
    r->t_setup_s = std::chrono::duration<double>(t0 - t_all).count();
    s = assemble_dev(ctx, g, kext.real(), kext.imag(), kint.real(), kint.imag(), eta_e, eta_i, p->asm_flags, 2,
                     dZ.p, n, nullptr, nullptr);
    if (s == BEM_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess)
        s = fail(ctx, BEM_ERR_CUDA, "assembly: %s", cudaGetErrorString(cudaGetLastError()));
    r->t_assembly_s = secs(t0);
    auto t1 = std::chrono::steady_clock::now();
    bem_lu* lu = nullptr;       // LU of Z, or of A_ext (GMRES preconditioner)
    bem_precond* M = nullptr;
    int info = 0;
    if (gm) {
        // A_ext = [[eta L_ext, -K_ext], [K_ext, L_ext/eta]] and its LU
        // (build_aext_preconditioner, bem_core.py:1071-1090); the
        // preconditioner's factorisation needs no int8 digit planes
        if (s == BEM_OK)
            s = assemble_dev(ctx, g, kext.real(), kext.imag(), 0, 0, eta_e, 1, p->asm_flags, 3, dA.p, n, nullptr,
                             nullptr);
        const int digits = ctx->oz_digits;
        ctx->oz_digits = 0;
        if (s == BEM_OK) s = bem_lu_factor_dev(ctx, dA.p, n, n, p->precision, &lu, &info);
        ctx->oz_digits = digits;
        if (s == BEM_OK && info > 0) s = fail(ctx, BEM_ERR_SINGULAR, "A_ext: zero pivot at %d", info);
        if (s == BEM_OK) s = bem_precond_create(ctx, BEM_PRECOND_LU, nullptr, n, n, p->precision, lu, &M);
    } else {
        if (s == BEM_OK) s = bem_lu_factor_dev(ctx, dZ.p, n, n, p->precision, &lu, &info);
        if (s == BEM_OK && info > 0) s = fail(ctx, BEM_ERR_SINGULAR, "zero pivot at %d", info);
    }
    const double gtol = p->gmres_tol > 0 ? p->gmres_tol : 1e-5;
    const int grestart = p->gmres_restart > 0 ? p->gmres_restart : std::min(200, n);
    const int gmaxiter = p->gmres_maxiter > 0 ? p->gmres_maxiter : 200;
    std::memset(&r->gmres, 0, sizeof r->gmres);
    r->gmres.converged = 1;
    r->t_solve_s = secs(t1);
    r->t_farfield_s = 0.0;
    // streamed multi-RHS solve and far field per batch
    std::vector<double> Mavg((size_t)16 * nt, 0.0), Mb((size_t)16 * nt), Mo;
    const double k2 = std::norm(kext);
    double w_sum = 0.0, w_total = 0.0, prev_csca = 0.0;
    for (double x : w) w_total += x;
    bool has_prev = false, converged = false;
    int consecutive_ok = 0, done = 0;
    std::memset(&r->stats, 0, sizeof r->stats);
    for (int o0 = 0; s == BEM_OK && o0 < no; o0 += batch) {
        const int nb = std::min(batch, no - o0), nrhs = 2 * nb;
        auto ts = std::chrono::steady_clock::now();
        s = rhs_dev(ctx, g, kext.real(), kext.imag(), eta_e, RT.data() + 9 * (size_t)o0, nullptr, nullptr, nb, dB.p,
                    n);
        bem_solve_stats st;
        std::memset(&st, 0, sizeof st);
        if (gm) {
            bem_gmres_stats gs;
            if (s == BEM_OK)
                s = bem_gmres_solve_dev(ctx, dZ.p, n, n, M, dB.p, n, dX.p, n, nrhs, grestart, gtol, gmaxiter, nullptr,
                                        nullptr, &gs);
            if (s != BEM_OK) break;
            bem_gmres_stats& a = r->gmres;
            a.converged = a.converged && gs.converged;
            a.n_unconverged += gs.n_unconverged;
            a.max_iterations = std::max(a.max_iterations, gs.max_iterations);
            a.total_iterations += gs.total_iterations;
            a.max_cycles = std::max(a.max_cycles, gs.max_cycles);
            a.matvecs += gs.matvecs;
            a.max_rel_residual = std::max(a.max_rel_residual, gs.max_rel_residual);
            a.t_ms += gs.t_ms;
            st.iterations = gs.max_iterations;
            st.converged = gs.converged;
            st.max_rel_residual = gs.max_rel_residual;
            st.t_factor_ms = 0;
            st.factorization = -1;
        } else if (s == BEM_OK) {
            s = bem_lu_solve_dev(ctx, lu, dB.p, n, dX.p, n, nrhs, p->refine_tol, p->max_refine, &st);
        }
        if (s != BEM_OK) break;
        r->stats.iterations = std::max(r->stats.iterations, st.iterations);
        r->stats.converged = o0 == 0 ? st.converged : (r->stats.converged && st.converged);
        r->stats.max_rel_update = std::max(r->stats.max_rel_update, st.max_rel_update);
        r->stats.max_rel_residual = std::max(r->stats.max_rel_residual, st.max_rel_residual);
        r->stats.est_rel_error = std::max(r->stats.est_rel_error, st.est_rel_error);
        r->stats.t_factor_ms = st.t_factor_ms;
        r->stats.t_solve_ms += st.t_solve_ms;
        r->stats.t_refine_ms += st.t_refine_ms;
        r->stats.factorization = st.factorization;
        r->stats.verified_columns += st.verified_columns;
        r->stats.verified_rel_error = std::max(r->stats.verified_rel_error, st.verified_rel_error);
        r->stats.exact_residual_sweeps = std::max(r->stats.exact_residual_sweeps, st.exact_residual_sweeps);
        for (int i = 0; i < 12; i++) r->stats.update_hist[i] = std::max(r->stats.update_hist[i], st.update_hist[i]);
        r->t_solve_s += secs(ts);
        auto tf = std::chrono::steady_clock::now();
        s = mueller_dev(ctx, g, dX.p, n, RT.data() + 9 * (size_t)o0, w.data() + o0, nb, kext.real(), kext.imag(),
                        eta_e, nt, p->gamma_mirror, Mb.data(), (double*)dMo.p);
        if (s != BEM_OK) break;
        for (size_t i = 0; i < Mb.size(); i++) Mavg[i] += Mb[i];
        if (r->per_orient_mueller || r->per_orient_weight) {
            Mo.resize((size_t)nb * 16 * nt);
            s = d2h(ctx, Mo.data(), dMo.p, Mo.size() * 8);
            if (s != BEM_OK) break;
            for (int o = 0; o < nb; o++) {
                const double wo = w[o0 + o];
                if (r->per_orient_weight) r->per_orient_weight[o0 + o] = wo;
                if (r->per_orient_mueller)
                    for (int i = 0; i < 16 * nt; i++)
                        r->per_orient_mueller[(size_t)(o0 + o) * 16 * nt + i] =
                            wo != 0.0 ? Mo[(size_t)o * 16 * nt + i] * k2 / wo : 0.0;
            }
        }
        r->t_farfield_s += secs(tf);
        done += nb;
        for (int o = 0; o < nb; o++) w_sum += w[o0 + o];
        // adaptive check (main.cpp:579-620)
        if (adaptive && done >= 40 && done % batch == 0) {
            double csca = 0.0;
            for (int it = 3; it < nt - 3; it++) csca += (Mavg[it] / w_sum) * std::sin(M_PI * it / (nt - 1));
            if (!has_prev) {
                prev_csca = csca;
                has_prev = true;
            } else {
                const double rel = std::abs(prev_csca) > 1e-30 ? std::abs(csca - prev_csca) / std::abs(prev_csca) : 0;
                consecutive_ok = rel < p->orient_tol ? consecutive_ok + 1 : 0;
                prev_csca = csca;
                if (consecutive_ok >= 2) {
                    converged = true;
                    break;
                }
            }
        }
    }
    auto tr = std::chrono::steady_clock::now();
    if (M) bem_precond_free(M);
    if (lu) bem_lu_free(lu);
    r->t_release_s = secs(tr);
    if (s == BEM_OK) {
        // rescale to the full weight after an early stop (main.cpp:624-636)
        const double scale = converged && done < no && w_sum > 0 ? w_total / w_sum : 1.0;
        for (size_t i = 0; i < Mavg.size(); i++) r->mueller[i] = Mavg[i] * scale;
    }
    r->n_computed = done;
    {
        auto tf = std::chrono::steady_clock::now();
        dZ.release();
        dB.release();
        dX.release();
        dMo.release();
        dA.release();
        bem_geom_free(g);
        g = nullptr;
        r->t_release_s += secs(tf);
    }
    r->t_total_s = secs(t_all);
    r->N = N;
    r->n_orient = no;
    bem_geom_free(g);
    return s;
}

}  // extern "C"

namespace {

// A bucket of FP64 particles with the same system size: every particle's
// operator assembled into one batch, one batched LU and one batched solve of
// all their right-hand sides (each launch covers the whole bucket), then the
// far field / Mueller matrix of each.  The batched LU is the blocked LU of the
// single path step for step (bitwise the same factors with the default shape).
int run_fp64_bucket(bem_ctx* ctx, const bem_problem* problems, const std::vector<int>& idx, bem_result* results,
                    int* statuses) {
    auto t_all = std::chrono::steady_clock::now();
    const int cnt = (int)idx.size();
    std::vector<bem_geom*> gs(cnt, nullptr);
    std::vector<std::vector<double>> RTs(cnt), ws(cnt);
    int n = 0, nrhs = 0, s = BEM_OK;
    for (int i = 0; i < cnt && s == BEM_OK; i++) {
        const bem_problem* p = &problems[idx[i]];
        int N = 0;
        s = bem_geom_create(ctx, p->verts, p->nv, p->tris, p->nt, p->quad_order, &gs[i], &N);
        if (s != BEM_OK) break;
        n = 2 * N;
        if (p->single) {
            RTs[i] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
            ws[i] = {1.0};
        } else {
            orientations(p->n_alpha, p->n_beta, p->n_gamma, p->beta_sym < 1 ? 1 : p->beta_sym,
                         p->gamma_sym < 1 ? 1 : p->gamma_sym, p->gamma_mirror != 0, true, RTs[i], ws[i]);
        }
        nrhs = std::max(nrhs, 2 * (int)ws[i].size());
    }
    const size_t nn = (size_t)n * n, nb = (size_t)n * nrhs;
    DevBuf dZ, dB, dX, dP;
    if (s == BEM_OK && (!dZ.alloc(ctx, nn * cnt * 16) || !dB.alloc(ctx, nb * cnt * 16) ||
                        !dX.alloc(ctx, nb * cnt * 16) || !dP.alloc(ctx, ((size_t)2 * n * cnt + cnt) * sizeof(int)))) {
        cudaGetLastError();
        s = fail(ctx, BEM_ERR_OOM, "bucket of %d particles of order %d", cnt, n);
    }
    double t_asm = 0, t_solve = 0, t_ff = 0;
    LuShape shape;
    if (s == BEM_OK && ctx->lu_autotune) s = tune_lu_shape(ctx, n, cnt, &shape);
    auto t0 = std::chrono::steady_clock::now();
    for (int i = 0; i < cnt && s == BEM_OK; i++) {
        const bem_problem* p = &problems[idx[i]];
        const std::complex<double> m(p->m_re, p->m_im), kext(p->ka, 0.0), kint = kext * m;
        s = assemble_dev(ctx, gs[i], kext.real(), kext.imag(), kint.real(), kint.imag(), 1.0, 1.0 / std::abs(m),
                         p->asm_flags, 2, (double2*)dZ.p + nn * i, n, nullptr, nullptr);
    }
    if (s == BEM_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess)
        s = fail(ctx, BEM_ERR_CUDA, "bucket assembly: %s", cudaGetErrorString(cudaGetLastError()));
    t_asm = secs(t0);
    auto t1 = std::chrono::steady_clock::now();
    int* d_ipiv = (int*)dP.p;
    int* d_perm = d_ipiv + (size_t)n * cnt;
    int* d_info = d_perm + (size_t)n * cnt;
    std::vector<int> info(cnt, 0), piv((size_t)n * cnt), perm;
    if (s == BEM_OK) s = getrf_batched(ctx, (double2*)dZ.p, n, (int64_t)nn, n, cnt, d_ipiv, d_info, shape);
    if (s == BEM_OK) s = d2h(ctx, info.data(), d_info, cnt * sizeof(int));
    if (s == BEM_OK) {
        int h_st = 0;
        s = d2h(ctx, &h_st, ctx->d_status, sizeof(int));
        if (s == BEM_OK && h_st != 0) s = fail(ctx, h_st, "device-side wait in the batched panel factorisation");
    }
    if (s == BEM_OK) s = d2h(ctx, piv.data(), d_ipiv, piv.size() * sizeof(int));
    if (s == BEM_OK) {
        std::vector<int> all((size_t)n * cnt);
        for (int i = 0; i < cnt; i++) {
            std::vector<int> pv(piv.begin() + (size_t)n * i, piv.begin() + (size_t)n * (i + 1));
            pivots_to_perm(pv, perm);
            std::copy(perm.begin(), perm.end(), all.begin() + (size_t)n * i);
        }
        s = h2d(ctx, d_perm, all.data(), all.size() * sizeof(int));
    }
    if (s == BEM_OK) {
        BEM_TRY_CUDA(ctx, cudaMemsetAsync(dB.p, 0, nb * cnt * 16, ctx->stream));
        for (int i = 0; i < cnt && s == BEM_OK; i++) {
            const bem_problem* p = &problems[idx[i]];
            s = rhs_dev(ctx, gs[i], p->ka, 0.0, 1.0, RTs[i].data(), nullptr, nullptr, (int)ws[i].size(),
                        (double2*)dB.p + nb * i, n);
        }
    }
    if (s == BEM_OK)
        s = getrs_batched(ctx, (const double2*)dZ.p, n, (int64_t)nn, n, cnt, d_perm, (const double2*)dB.p, n,
                          (int64_t)nb, (double2*)dX.p, n, (int64_t)nb, nrhs, shape.NB);
    if (s == BEM_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess)
        s = fail(ctx, BEM_ERR_CUDA, "bucket solve: %s", cudaGetErrorString(cudaGetLastError()));
    t_solve = secs(t1);
    auto t2 = std::chrono::steady_clock::now();
    for (int i = 0; i < cnt; i++) {
        const bem_problem* p = &problems[idx[i]];
        bem_result* r = &results[idx[i]];
        int si = s;
        if (si == BEM_OK && info[i] > 0) si = fail(ctx, BEM_ERR_SINGULAR, "particle %d: zero pivot at %d", idx[i], info[i]);
        if (si == BEM_OK) {
            const int no = (int)ws[i].size(), nt = p->ntheta;
            std::vector<double> M((size_t)16 * nt);
            si = mueller_dev(ctx, gs[i], (double2*)dX.p + nb * i, n, RTs[i].data(), ws[i].data(), no, p->ka, 0.0, 1.0,
                             nt, p->gamma_mirror, M.data(), nullptr);
            if (si == BEM_OK) std::memcpy(r->mueller, M.data(), M.size() * 8);
            r->N = n / 2;
            r->n_orient = no;
            r->n_computed = no;
            std::memset(&r->stats, 0, sizeof r->stats);
            r->stats.converged = 1;
            r->stats.factorization = -1;
        }
        if (statuses) statuses[idx[i]] = si;
    }
    t_ff = secs(t2);
    for (int i = 0; i < cnt; i++) {
        bem_result* r = &results[idx[i]];
        // the bucket's phase times, shared equally by its particles
        r->t_assembly_s = t_asm / cnt;
        r->t_solve_s = t_solve / cnt;
        r->t_farfield_s = t_ff / cnt;
        r->t_total_s = secs(t_all) / cnt;
        if (gs[i]) bem_geom_free(gs[i]);
    }
    return s;
}

}  // namespace

extern "C" {

// Batched particles.  FP64 particles of one system size (without adaptive
// orientation stopping, GMRES or per-orientation output) go through
// run_fp64_bucket: one batched assembly pass, batched LU and batched solve per
// size, with the LU's block / panel shape chosen by the autotuner; the others
// through the dense pipeline in turn.  statuses[i] (optional) receives each
// problem's status; a failing particle does not stop the batch.  Returns
// BEM_OK, or the first failure.  (Worker contexts on several streams were
// measured slower: the persistent tensor-core kernels take one CTA per SM and
// do not overlap.)
int bem_batch_run(bem_ctx* ctx, const bem_problem* problems, int count, bem_result* results, int* statuses) {
    if (!ctx || count < 0 || (count > 0 && (!problems || !results))) return BEM_ERR_INVALID;
    // particles of one topology reuse their device buffers (operator,
    // right-hand sides, factors, digit planes, geometry) through the device-
    // memory cache for the duration of the batch; it is released at the end
    // unless the caller keeps it on (cache_factor_memory)
    const bool had_cache = devmem_cache_enabled(ctx->device);
    if (!had_cache) devmem_cache_enable(ctx->device, true);
    int first = BEM_OK;
    std::string first_msg;
    std::vector<int> st(count, BEM_OK);
    std::vector<char> done(count, 0);
    if (ctx->batch_buckets) {
        // FP64 particles grouped by system size (2N from the mesh's RWG count)
        std::map<int, std::vector<int>> buckets;
        for (int i = 0; i < count; i++) {
            const bem_problem& p = problems[i];
            if (p.precision != BEM_PREC_FP64 || p.solver != BEM_SOLVER_LU || p.orient_tol > 0 ||
                results[i].per_orient_mueller || results[i].per_orient_weight || !results[i].mueller ||
                !(p.ka > 0) || p.ntheta < 2 || (!p.single && p.orient_i0 >= 0))
                continue;
            HostMesh hm;
            if (!host_mesh_from(p.verts, p.nv, p.tris, p.nt, &hm)) continue;
            buckets[build_rwg(hm).N].push_back(i);
        }
        for (auto& kv : buckets) {
            if (kv.second.size() < 2) continue;
            std::vector<int> sts(count, BEM_OK);
            run_fp64_bucket(ctx, problems, kv.second, results, sts.data());
            for (int i : kv.second) st[i] = sts[i], done[i] = 1;
        }
    }
    for (int i = 0; i < count; i++) {
        if (!done[i]) st[i] = bem_dense_run(ctx, &problems[i], &results[i]);
        if (statuses) statuses[i] = st[i];
        if (st[i] != BEM_OK && first == BEM_OK) {
            first = st[i];
            first_msg = "particle " + std::to_string(i) + ": " + ctx->last_error;
        }
    }
    if (!had_cache) devmem_cache_enable(ctx->device, false);
    if (first != BEM_OK) ctx->last_error = first_msg;
    return first;
}

}  // extern "C"
