// A consumer of the reference's C++ call surface (include/bem/*.h over
// libbem_compat.so): the calls of the reference's dense branch
// (main.cpp:660-854) in their call forms -- mesh, RWG, far-field cache,
// assemble_pmchwt with NULL L_ext / K_ext, lu_factorize_cuda + lu_solve_cuda
// for one orientation, compute_rhs_planewave per polarisation, lu_solve_full
// for many, compute_far_field, FFCacheGPU + compute_farfield_batch_cuda,
// amplitude_to_mueller and write_json.
//
// Usage: dense_branch OUTDIR [REF KA M_RE M_IM NA NB NG NTHETA [AR]]
// (defaults: icosphere refinement 1, ka 1, m 1.3116, 2 x 2 x 1 orientations,
// 19 angles; AR > 0: the hexagonal prism of that aspect ratio instead of the
// icosphere).  The same source builds against the reference's own headers
// and sources (its dense path: FP32 assembly kernel, cuSOLVER), which is how
// the reference's GPU path is timed beside this library's.  Writes into
// OUTDIR, for the tests to compare:
//   Z.bin        assemble_pmchwt's Z (row-major 2N x 2N complex128)
//   B1.bin       the single orientation's right-hand sides (k = z, E = x / y)
//   X1.bin       their solution by lu_factorize_cuda + lu_solve_cuda
//   ipiv.bin     lu_factorize_cuda's pivots (1-based int32)
//   Xfull1.bin   the same right-hand sides through lu_solve_full
//   Xo.bin       every orientation's solution through lu_solve_full
//   Fsingle.bin  compute_far_field of the single orientation's x column (F_theta, F_phi)
//   single.json  the single orientation's Mueller matrix (batched far field), write_json
//   orient.json  the orientation-averaged Mueller matrix, write_json
//   singular.txt lu_factorize_cuda's info and lu_solve_full's status on Z with
//                row and column N (0-based) zeroed (expected info N + 1)
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "mesh.h"
#include "rwg.h"
#include "quadrature.h"
#include "pmchwt.h"
#include "solver.h"
#include "rhs.h"
#include "farfield.h"
#include "orient.h"
#include "output.h"

using cd = std::complex<double>;

static bool dump(const std::string& path, const void* p, size_t bytes) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    bool ok = std::fwrite(p, 1, bytes, f) == bytes;
    return std::fclose(f) == 0 && ok;
}

// Batched far field of n_calls = 2 no solution columns (par, perp per
// orientation) and the weighted Mueller sum (main.cpp:757-846).
static std::vector<double> mueller_of(const RWG& rwg, const FFCache& ff_cache, const std::vector<cd>& X, int N2,
                                      const std::vector<Orientation>& orients, cd k_ext, double eta_ext,
                                      const std::vector<double>& theta) {
    const int N = rwg.N, no = (int)orients.size(), n_calls = 2 * no, ntheta = (int)theta.size();
    FFCacheGPU ff_gpu;
    ff_gpu.upload(ff_cache);
    std::vector<cd> cJ(n_calls * N), cM(n_calls * N);
    for (int c = 0; c < n_calls; c++)
        for (int n = 0; n < N; n++) {
            cJ[c * N + n] = X[c * N2 + n];
            cM[c * N + n] = X[c * N2 + N + n];
        }
    std::vector<double> r_hats(no * ntheta * 3);
    std::vector<Vec3> e_par(no * ntheta), e_perp(no * ntheta);
    for (int o = 0; o < no; o++)
        for (int t = 0; t < ntheta; t++) {
            const double ct = std::cos(theta[t]), st = std::sin(theta[t]);
            const Vec3 rh = orients[o].RT * Vec3(st, 0, ct);
            r_hats[(o * ntheta + t) * 3] = rh.x;
            r_hats[(o * ntheta + t) * 3 + 1] = rh.y;
            r_hats[(o * ntheta + t) * 3 + 2] = rh.z;
            e_par[o * ntheta + t] = orients[o].RT * Vec3(ct, 0, -st);
            e_perp[o * ntheta + t] = orients[o].RT * Vec3(0, 1, 0);
        }
    std::vector<cd> Fv(n_calls * ntheta * 3);
    compute_farfield_batch_cuda(ff_gpu, cJ.data(), cM.data(), r_hats.data(), k_ext, eta_ext, n_calls, no, ntheta,
                                Fv.data());
    ff_gpu.free();
    const cd mik = cd(0, -1) * k_ext;
    const double k2 = std::norm(k_ext);
    std::vector<double> M_avg(16 * ntheta, 0.0), M_o(16 * ntheta);
    for (int o = 0; o < no; o++) {
        std::vector<cd> S1(ntheta), S2(ntheta), S3(ntheta), S4(ntheta);
        for (int t = 0; t < ntheta; t++) {
            const cd* a = &Fv[((2 * o) * ntheta + t) * 3];
            const cd* b = &Fv[((2 * o + 1) * ntheta + t) * 3];
            const Vec3 &ep = e_par[o * ntheta + t], &epp = e_perp[o * ntheta + t];
            S2[t] = mik * (a[0] * ep.x + a[1] * ep.y + a[2] * ep.z);
            S4[t] = mik * (a[0] * epp.x + a[1] * epp.y + a[2] * epp.z);
            S3[t] = mik * (b[0] * ep.x + b[1] * ep.y + b[2] * ep.z);
            S1[t] = mik * (b[0] * epp.x + b[1] * epp.y + b[2] * epp.z);
        }
        amplitude_to_mueller(S1.data(), S2.data(), S3.data(), S4.data(), ntheta, M_o.data());
        for (int i = 0; i < 16 * ntheta; i++) M_avg[i] += orients[o].weight * M_o[i] / k2;
    }
    return M_avg;
}

int main(int argc, char** argv) {
    const std::string out = argc > 1 ? argv[1] : ".";
    const int ref = argc > 2 ? std::atoi(argv[2]) : 1;
    const double ka = argc > 3 ? std::atof(argv[3]) : 1.0;
    const double n_re = argc > 4 ? std::atof(argv[4]) : 1.3116, n_im = argc > 5 ? std::atof(argv[5]) : 0.0;
    const int na = argc > 6 ? std::atoi(argv[6]) : 2, nb = argc > 7 ? std::atoi(argv[7]) : 2,
              ng = argc > 8 ? std::atoi(argv[8]) : 1, ntheta = argc > 9 ? std::atoi(argv[9]) : 19;
    const double ar = argc > 10 ? std::atof(argv[10]) : 0.0;
    const int quad = 7;
    Mesh mesh = ar > 0 ? hex_prism(ar, ref) : icosphere(1.0, ref);
    RWG rwg = build_rwg(mesh);
    const int N = rwg.N, N2 = 2 * N;
    const cd k_ext(ka, 0.0), k_int = k_ext * cd(n_re, n_im);
    const double eta_ext = 1.0, eta_int = 1.0 / std::abs(cd(n_re, n_im));
    FFCache ff_cache;
    ff_cache.init(rwg, mesh, quad);
    std::vector<double> theta(ntheta);
    for (int t = 0; t < ntheta; t++) theta[t] = M_PI * t / (ntheta - 1);
    {
        // device and library start-up outside the timed phases: a small assembly
        Mesh m0 = icosphere(1.0, 0);
        RWG r0 = build_rwg(m0);
        std::vector<cd> Z0((size_t)4 * r0.N * r0.N);
        assemble_pmchwt(r0, m0, k_ext, k_int, eta_ext, eta_int, quad, Z0.data(), NULL, NULL);
    }

    Timer asm_timer;
    std::vector<cd> Z((size_t)N2 * N2), Zc;
    assemble_pmchwt(rwg, mesh, k_ext, k_int, eta_ext, eta_int, quad, Z.data(), NULL, NULL);
    const double t_asm = asm_timer.elapsed_s();
    if (!dump(out + "/Z.bin", Z.data(), Z.size() * sizeof(cd))) return 10;
    Zc = Z;

    // one orientation (--single): factor once, two polarisations
    std::vector<int> ipiv(N2);
    if (lu_factorize_cuda(Zc.data(), N2, ipiv.data()) != 0) return 2;
    std::vector<cd> B(N2 * 2);
    compute_rhs_planewave(rwg, mesh, k_ext, eta_ext, Vec3(1, 0, 0), Vec3(0, 0, 1), quad, &B[0]);
    compute_rhs_planewave(rwg, mesh, k_ext, eta_ext, Vec3(0, 1, 0), Vec3(0, 0, 1), quad, &B[N2]);
    std::vector<cd> X1 = B;
    if (lu_solve_cuda(Zc.data(), ipiv.data(), N2, X1.data(), 2) != 0) return 3;
    std::vector<cd> Fth(ntheta), Fph(ntheta);
    compute_far_field(ff_cache, &X1[0], &X1[N], k_ext, eta_ext, theta.data(), ntheta, Fth.data(), Fph.data());
    std::vector<cd> Xf = B, Zs = Z;
    if (lu_solve_full(Zs.data(), N2, Xf.data(), 2) != 0) return 4;
    std::vector<cd> F(2 * ntheta);
    for (int t = 0; t < ntheta; t++) F[t] = Fth[t], F[ntheta + t] = Fph[t];
    if (!dump(out + "/B1.bin", B.data(), B.size() * sizeof(cd)) ||
        !dump(out + "/X1.bin", X1.data(), X1.size() * sizeof(cd)) ||
        !dump(out + "/ipiv.bin", ipiv.data(), ipiv.size() * sizeof(int)) ||
        !dump(out + "/Xfull1.bin", Xf.data(), Xf.size() * sizeof(cd)) ||
        !dump(out + "/Fsingle.bin", F.data(), F.size() * sizeof(cd)))
        return 11;
    std::vector<Orientation> single(1);
    single[0].RT = euler_rotation(0.0, 0.0, 0.0);
    single[0].weight = 1.0;
    std::vector<double> M1 = mueller_of(rwg, ff_cache, X1, N2, single, k_ext, eta_ext, theta);
    write_json((out + "/single.json").c_str(), M1.data(), theta.data(), ntheta, ka, n_re, n_im, ref, 1, 1, 1, t_asm,
               0.0, 0.0, t_asm);

    // orientation average: all right-hand sides, one lu_solve_full, batched far field
    Timer solve_timer;
    std::vector<Orientation> orients = generate_orientations(na, nb, ng);
    const int no = (int)orients.size(), n_calls = 2 * no;
    std::vector<cd> Bo((size_t)N2 * n_calls);
    for (int o = 0; o < no; o++) {
        const Mat3& RT = orients[o].RT;
        compute_rhs_planewave(rwg, mesh, k_ext, eta_ext, RT * Vec3(1, 0, 0), RT * Vec3(0, 0, 1), quad,
                              &Bo[(2 * o) * N2]);
        compute_rhs_planewave(rwg, mesh, k_ext, eta_ext, RT * Vec3(0, 1, 0), RT * Vec3(0, 0, 1), quad,
                              &Bo[(2 * o + 1) * N2]);
    }
    const double t_rhs = solve_timer.elapsed_s();
    Zs = Z;
    if (lu_solve_full(Zs.data(), N2, Bo.data(), n_calls) != 0) return 5;
    const double t_solve = solve_timer.elapsed_s();
    if (!dump(out + "/Xo.bin", Bo.data(), Bo.size() * sizeof(cd))) return 12;
    Timer ff_timer;
    std::vector<double> M_avg = mueller_of(rwg, ff_cache, Bo, N2, orients, k_ext, eta_ext, theta);
    const double t_ff = ff_timer.elapsed_s();
    write_json((out + "/orient.json").c_str(), M_avg.data(), theta.data(), ntheta, ka, n_re, n_im, ref, na, nb, ng,
               t_asm, t_solve, t_ff, t_asm + t_solve + t_ff);

    // a singular matrix: row and column N zeroed; the LU reports the zero
    // pivot (LAPACK info, 1-based) and lu_solve_full fails
    Zs = Z;
    for (int i = 0; i < N2; i++) Zs[(size_t)N * N2 + i] = Zs[(size_t)i * N2 + N] = 0.0;
    std::vector<cd> Zs2 = Zs, Bs = B;
    const int info = lu_factorize_cuda(Zs.data(), N2, ipiv.data());
    const int full = lu_solve_full(Zs2.data(), N2, Bs.data(), 2);
    FILE* f = std::fopen((out + "/singular.txt").c_str(), "w");
    if (!f) return 13;
    std::fprintf(f, "%d %d\n", info, full);
    std::fclose(f);
    std::printf("single-orientation |F_theta(0)| = %.6e\n", std::abs(Fth[0]));
    std::printf("phase seconds: assembly %.6f rhs %.6f lu_solve_full %.6f farfield+mueller %.6f\n", t_asm, t_rhs,
                t_solve - t_rhs, t_ff);
    return 0;
}
