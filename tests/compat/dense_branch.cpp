// A consumer of the reference's C++ call surface (include/bem/*.h over
// libbem_compat.so): the calls of the reference's dense branch
// (main.cpp:660-854) in their call forms -- mesh, RWG, far-field cache,
// assemble_pmchwt with NULL L_ext / K_ext, lu_factorize_cuda + lu_solve_cuda
// for one orientation, compute_rhs_planewave per polarisation, lu_solve_full
// for many, compute_far_field, FFCacheGPU + compute_farfield_batch_cuda,
// amplitude_to_mueller and write_json.  Built on the CPU by the tests to
// show that the surface accepts those forms; it runs only with a GPU.
#include <cmath>
#include <complex>
#include <cstdio>
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

int main(int argc, char** argv) {
    const char* out = argc > 1 ? argv[1] : "compat_result.json";
    const double ka = 1.0, n_re = 1.3116, n_im = 0.0;
    const int ref = 1, quad = 7, ntheta = 19, na = 2, nb = 2, ng = 1;
    Mesh mesh = icosphere(1.0, ref);
    RWG rwg = build_rwg(mesh);
    const int N = rwg.N, N2 = 2 * N;
    const std::complex<double> k_ext(ka, 0.0), k_int = k_ext * std::complex<double>(n_re, n_im);
    const double eta_ext = 1.0, eta_int = 1.0 / std::abs(std::complex<double>(n_re, n_im));
    FFCache ff_cache;
    ff_cache.init(rwg, mesh, quad);
    std::vector<double> theta(ntheta);
    for (int t = 0; t < ntheta; t++) theta[t] = M_PI * t / (ntheta - 1);

    Timer asm_timer;
    std::vector<std::complex<double>> Z(N2 * N2), Zc;
    assemble_pmchwt(rwg, mesh, k_ext, k_int, eta_ext, eta_int, quad, Z.data(), NULL, NULL);
    const double t_asm = asm_timer.elapsed_s();
    Zc = Z;

    // one orientation: factor once, two polarisations, the phi = 0 plane
    std::vector<int> ipiv(N2);
    if (lu_factorize_cuda(Zc.data(), N2, ipiv.data()) != 0) return 2;
    std::vector<std::complex<double>> B(N2 * 2);
    compute_rhs_planewave(rwg, mesh, k_ext, eta_ext, Vec3(1, 0, 0), Vec3(0, 0, 1), quad, &B[0]);
    compute_rhs_planewave(rwg, mesh, k_ext, eta_ext, Vec3(0, 1, 0), Vec3(0, 0, 1), quad, &B[N2]);
    if (lu_solve_cuda(Zc.data(), ipiv.data(), N2, B.data(), 2) != 0) return 3;
    std::vector<std::complex<double>> Fth(ntheta), Fph(ntheta);
    compute_far_field(ff_cache, &B[0], &B[N], k_ext, eta_ext, theta.data(), ntheta, Fth.data(), Fph.data());

    // orientation average: all right-hand sides, one solve, batched far field
    Timer solve_timer;
    std::vector<Orientation> orients = generate_orientations(na, nb, ng);
    const int no = (int)orients.size(), n_calls = 2 * no;
    std::vector<std::complex<double>> Bo(N2 * n_calls);
    for (int o = 0; o < no; o++) {
        const Mat3& RT = orients[o].RT;
        compute_rhs_planewave(rwg, mesh, k_ext, eta_ext, RT * Vec3(1, 0, 0), RT * Vec3(0, 0, 1), quad,
                              &Bo[(2 * o) * N2]);
        compute_rhs_planewave(rwg, mesh, k_ext, eta_ext, RT * Vec3(0, 1, 0), RT * Vec3(0, 0, 1), quad,
                              &Bo[(2 * o + 1) * N2]);
    }
    if (lu_solve_full(Z.data(), N2, Bo.data(), n_calls) != 0) return 4;
    const double t_solve = solve_timer.elapsed_s();

    Timer ff_timer;
    FFCacheGPU ff_gpu;
    ff_gpu.upload(ff_cache);
    std::vector<std::complex<double>> cJ(n_calls * N), cM(n_calls * N);
    for (int c = 0; c < n_calls; c++)
        for (int n = 0; n < N; n++) {
            cJ[c * N + n] = Bo[c * N2 + n];
            cM[c * N + n] = Bo[c * N2 + N + n];
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
    std::vector<std::complex<double>> Fv(n_calls * ntheta * 3);
    compute_farfield_batch_cuda(ff_gpu, cJ.data(), cM.data(), r_hats.data(), k_ext, eta_ext, n_calls, no, ntheta,
                                Fv.data());
    const std::complex<double> mik = std::complex<double>(0, -1) * k_ext;
    const double k2 = std::norm(k_ext);
    std::vector<double> M_avg(16 * ntheta, 0.0), M_o(16 * ntheta);
    for (int o = 0; o < no; o++) {
        std::vector<std::complex<double>> S1(ntheta), S2(ntheta), S3(ntheta), S4(ntheta);
        for (int t = 0; t < ntheta; t++) {
            const std::complex<double>* a = &Fv[((2 * o) * ntheta + t) * 3];
            const std::complex<double>* b = &Fv[((2 * o + 1) * ntheta + t) * 3];
            const Vec3 &ep = e_par[o * ntheta + t], &epp = e_perp[o * ntheta + t];
            S2[t] = mik * (a[0] * ep.x + a[1] * ep.y + a[2] * ep.z);
            S4[t] = mik * (a[0] * epp.x + a[1] * epp.y + a[2] * epp.z);
            S3[t] = mik * (b[0] * ep.x + b[1] * ep.y + b[2] * ep.z);
            S1[t] = mik * (b[0] * epp.x + b[1] * epp.y + b[2] * epp.z);
        }
        amplitude_to_mueller(S1.data(), S2.data(), S3.data(), S4.data(), ntheta, M_o.data());
        for (int i = 0; i < 16 * ntheta; i++) M_avg[i] += orients[o].weight * M_o[i] / k2;
    }
    write_json(out, M_avg.data(), theta.data(), ntheta, ka, n_re, n_im, ref, na, nb, ng, t_asm, t_solve,
               ff_timer.elapsed_s(), t_asm + t_solve + ff_timer.elapsed_s());
    std::printf("single-orientation |F_theta(0)| = %.6e\n", std::abs(Fth[0]));
    return 0;
}
