// bem_cuda -- the --solver dense command line of BEM-CPP (main.cpp:25-181,
// dense branch :660-854) over libbemdense: same flags, same JSON output
// (output.cpp:5-64).  Assembly, factorisation, the solve of every
// orientation x polarisation and the far field / Mueller reduction run on the
// device through bem_dense_run.  Iterative-solver flags are accepted and
// ignored with a warning (bem_cuda provides the dense path only).
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "bem/mesh.h"
#include "bem/output.h"
#include "bem/rwg.h"
#include "bem_dense.h"

static void usage(const char* prog) {
    std::printf("Usage: %s [options]\n", prog);
    std::printf("  --ka F             Size parameter (required)\n");
    std::printf("  --ri RE IM         Refractive index (default: 1.3116 0)\n");
    std::printf("  --ref N            Refinement level (default: 3)\n");
    std::printf("  --orient NA NB NG  Orientation quadrature (default: 8 8 1)\n");
    std::printf("  --ntheta N         Number of scattering angles (default: 181)\n");
    std::printf("  --quad N           Quadrature order: 4, 7, 13 (default: 7)\n");
    std::printf("  --out FILE         Output JSON file (default: result.json)\n");
    std::printf("  --single           Single orientation (no averaging)\n");
    std::printf("  --solver TYPE      dense (default; auto selects dense)\n");
    std::printf("  --shape TYPE       sphere (default) or hex\n");
    std::printf("  --ar F             Hex aspect ratio H/D (default: 1.0)\n");
    std::printf("  --obj FILE         Load mesh from OBJ file\n");
    std::printf("  --subdiv N         Subdivide the OBJ mesh N times\n");
    std::printf("  --orient-sym B G   Orientation symmetry factors (default: 1 1)\n");
    std::printf("  --gamma-mirror     Gamma mirror symmetry\n");
    std::printf("  --orient-range I0 I1  Only orientations [I0, I1)\n");
    std::printf("  --orient-auto [R]  Orientation count from ka and D_max (default R=4)\n");
    std::printf("  --precision P      fp64 (default) or fp32-refine\n");
    std::printf("  --refine-tol F     FP32+refinement error target (default 1e-11)\n");
    std::printf("  --dense-solver S   lu (default) or gmres-aext: GMRES on Z preconditioned by\n");
    std::printf("                     the LU of the exterior-only A_ext (bem_core.py:1093)\n");
    std::printf("  --gmres-tol F      gmres-aext relative tolerance (default 1e-5)\n");
    std::printf("  --gmres-restart N  gmres-aext restart (default min(200, 2N))\n");
}

int main(int argc, char** argv) {
    setbuf(stdout, NULL);
    double ka = 0, n_re = 1.3116, n_im = 0.0, hex_ar = 1.0, refine_tol = 0.0, orient_auto_R = 4.0;
    double orient_tol = 0.0, gmres_tol = 0.0;
    int gmres_restart = 0, dense_solver = BEM_SOLVER_LU;
    int ref = 3, na = 8, nb = 8, ng = 1, ntheta = 181, quad = 7, bsym = 1, gsym = 1, i0 = -1, i1 = -1, subdiv = 0;
    bool single = false, mirror = false, orient_auto = false;
    int precision = BEM_PREC_FP64;
    std::string shape = "sphere";
    const char* out = "result.json";
    const char* obj = nullptr;
    for (int i = 1; i < argc; i++) {
        auto is = [&](const char* f, int nargs) { return std::strcmp(argv[i], f) == 0 && i + nargs < argc; };
        if (is("--ka", 1)) ka = std::atof(argv[++i]);
        else if (is("--ri", 2)) { n_re = std::atof(argv[++i]); n_im = std::atof(argv[++i]); }
        else if (is("--ref", 1)) ref = std::atoi(argv[++i]);
        else if (is("--orient", 3)) { na = std::atoi(argv[++i]); nb = std::atoi(argv[++i]); ng = std::atoi(argv[++i]); }
        else if (is("--ntheta", 1)) ntheta = std::atoi(argv[++i]);
        else if (is("--quad", 1)) quad = std::atoi(argv[++i]);
        else if (is("--out", 1)) out = argv[++i];
        else if (std::strcmp(argv[i], "--single") == 0) single = true;
        else if (is("--solver", 1)) {
            const char* s = argv[++i];
            if (std::strcmp(s, "dense") != 0 && std::strcmp(s, "auto") != 0) {
                std::fprintf(stderr, "Solver '%s' is not provided by bem_cuda (dense only)\n", s);
                return 1;
            }
        } else if (is("--shape", 1)) shape = argv[++i];
        else if (is("--ar", 1)) hex_ar = std::atof(argv[++i]);
        else if (is("--obj", 1)) obj = argv[++i];
        else if (is("--subdiv", 1)) subdiv = std::atoi(argv[++i]);
        else if (is("--orient-sym", 2)) { bsym = std::atoi(argv[++i]); gsym = std::atoi(argv[++i]); }
        else if (std::strcmp(argv[i], "--gamma-mirror") == 0) mirror = true;
        else if (is("--orient-range", 2)) { i0 = std::atoi(argv[++i]); i1 = std::atoi(argv[++i]); }
        else if (std::strcmp(argv[i], "--orient-auto") == 0) {
            orient_auto = true;
            if (i + 1 < argc && argv[i + 1][0] != '-') orient_auto_R = std::atof(argv[++i]);
        } else if (is("--precision", 1)) {
            const char* p = argv[++i];
            if (std::strcmp(p, "fp64") == 0) precision = BEM_PREC_FP64;
            else if (std::strcmp(p, "fp32-refine") == 0) precision = BEM_PREC_FP32_REFINE;
            else { std::fprintf(stderr, "Unknown precision: %s\n", p); return 1; }
        } else if (is("--refine-tol", 1)) refine_tol = std::atof(argv[++i]);
        else if (is("--orient-tol", 1)) orient_tol = std::atof(argv[++i]);
        else if (is("--dense-solver", 1)) {
            const char* d = argv[++i];
            if (std::strcmp(d, "lu") == 0) dense_solver = BEM_SOLVER_LU;
            else if (std::strcmp(d, "gmres-aext") == 0) dense_solver = BEM_SOLVER_GMRES_AEXT;
            else { std::fprintf(stderr, "Unknown dense solver: %s\n", d); return 1; }
        } else if (is("--gmres-tol", 1)) gmres_tol = std::atof(argv[++i]);
        else if (is("--gmres-restart", 1)) gmres_restart = std::atoi(argv[++i]);
        else if (is("--digits", 1) || is("--max-leaf", 1) ||
                 is("--prec", 1) || is("--prec-r", 1) || is("--prec-bs", 1) || is("--prec-overlap", 1)) {
            std::fprintf(stderr, "Warning: %s applies to the iterative solvers; ignored\n", argv[i]);
            ++i;
        } else if (std::strcmp(argv[i], "--goi") == 0) {
            std::fprintf(stderr, "Warning: --goi applies to the iterative solvers; ignored\n");
        } else if (std::strcmp(argv[i], "--help") == 0 || std::strcmp(argv[i], "-h") == 0) {
            usage(argv[0]);
            return 0;
        } else {
            std::fprintf(stderr, "Unknown option: %s\n", argv[i]);
            usage(argv[0]);
            return 1;
        }
    }
    if (ka <= 0) {
        std::fprintf(stderr, "Error: --ka must be positive\n");
        usage(argv[0]);
        return 1;
    }
    Timer total;
    Mesh mesh;
    if (obj) {
        mesh = load_obj(obj);
        double a = normalize_mesh(mesh);
        std::printf("  OBJ normalized: a_eq=%.4f, scaled to unit\n", a);
        for (int s = 0; s < subdiv; s++) mesh = subdivide_flat(mesh);
    } else if (shape == "hex") {
        mesh = hex_prism(hex_ar, ref);
    } else {
        mesh = icosphere(1.0, ref);
    }
    double dmax = mesh_dmax(mesh);
    if (orient_auto && !single) {
        // main.cpp:263-280
        double lambda = 2.0 * M_PI / ka;
        double xi_deg = 0.69 * lambda / dmax * (180.0 / M_PI);
        double delta = xi_deg / 3.0 * orient_auto_R;
        na = std::max(4, (int)std::ceil(360.0 / delta));
        nb = std::max(2, (int)std::ceil(180.0 / delta));
        ng = 1;
        if (na % 2 == 0) na++;
        if (nb % 2 == 0) nb++;
    }
    std::printf("=== BEM dense (sm_100a) ===\n  ka = %.4f, m = %.4f + %.4fi, %d vertices, %d triangles\n", ka, n_re, n_im,
                mesh.nv(), mesh.nt());
    bem_ctx* ctx = nullptr;
    const char* dev = std::getenv("BEM_DEVICE");
    int s = bem_ctx_create(dev ? std::atoi(dev) : 0, &ctx);
    if (s != BEM_OK) {
        std::fprintf(stderr, "No usable sm_100 device (status %d)\n", s);
        return 1;
    }
    std::vector<double> v(3 * (size_t)mesh.nv());
    for (int i = 0; i < mesh.nv(); i++) v[3 * i] = mesh.verts[i].x, v[3 * i + 1] = mesh.verts[i].y, v[3 * i + 2] = mesh.verts[i].z;
    bem_problem p;
    std::memset(&p, 0, sizeof p);
    p.verts = v.data();
    p.nv = mesh.nv();
    p.tris = mesh.tris.data();
    p.nt = mesh.nt();
    p.ka = ka;
    p.m_re = n_re;
    p.m_im = n_im;
    p.quad_order = (quad == 4 || quad == 13) ? quad : 7;
    p.single = single;
    p.n_alpha = na;
    p.n_beta = nb;
    p.n_gamma = ng;
    p.beta_sym = bsym;
    p.gamma_sym = gsym;
    p.gamma_mirror = mirror;
    p.orient_i0 = i0;
    p.orient_i1 = i1;
    p.ntheta = ntheta;
    p.precision = precision;
    p.refine_tol = refine_tol;
    p.orient_tol = orient_tol;
    p.solver = dense_solver;
    p.gmres_tol = gmres_tol;
    p.gmres_restart = gmres_restart;
    std::vector<double> M(16 * (size_t)ntheta), theta(ntheta);
    for (int t = 0; t < ntheta; t++) theta[t] = M_PI * t / (ntheta - 1);
    bem_result r;
    std::memset(&r, 0, sizeof r);
    r.mueller = M.data();
    // per-orientation stream of the adaptive mode (main.cpp:640-653)
    std::vector<double> po_M, po_w;
    if (orient_tol > 0 && !single) {
        int count = 0;
        bem_orientations(na, nb, ng, bsym, gsym, mirror, 1, &count, nullptr, nullptr);
        po_M.resize((size_t)count * 16 * ntheta);
        po_w.resize(count);
        r.per_orient_mueller = po_M.data();
        r.per_orient_weight = po_w.data();
    }
    s = bem_dense_run(ctx, &p, &r);
    if (s != BEM_OK) {
        std::fprintf(stderr, "Dense solve failed (status %d): %s\n", s, bem_last_error(ctx));
        bem_ctx_destroy(ctx);
        return 1;
    }
    std::printf("  RWG: %d basis functions, %d orientations\n", r.N, r.n_orient);
    if (orient_tol > 0 && !single) {
        std::printf("  Averaged over %d/%d orientations.\n", r.n_computed, r.n_orient);
        std::string po_path = std::string(out) + ".per_orient";
        if (FILE* pf = std::fopen(po_path.c_str(), "wb")) {
            int header[4] = {r.n_computed, ntheta, na, nb};
            std::fwrite(header, sizeof(int), 4, pf);
            std::fwrite(po_w.data(), sizeof(double), r.n_computed, pf);
            std::fwrite(po_M.data(), sizeof(double), (size_t)r.n_computed * 16 * ntheta, pf);
            std::fclose(pf);
            std::printf("  Per-orient Mueller saved: %s (%d orient x 16 x %d)\n", po_path.c_str(), r.n_computed,
                        ntheta);
        }
    }
    if (dense_solver == BEM_SOLVER_GMRES_AEXT)
        std::printf("  GMRES(A_ext): max %d iter per column, %d columns unconverged, max rel. residual %.2e\n",
                    r.gmres.max_iterations, r.gmres.n_unconverged, r.gmres.max_rel_residual);
    else if (precision == BEM_PREC_FP32_REFINE)
        std::printf("  FP32 + refinement: %d sweeps, estimated rel. error %.2e\n", r.stats.iterations,
                    r.stats.est_rel_error);
    write_json(out, M.data(), theta.data(), ntheta, ka, n_re, n_im, ref, na, nb, ng, r.t_assembly_s, r.t_solve_s,
               r.t_farfield_s, total.elapsed_s());
    std::printf("\n=== Done ===\n  Assembly: %.1fs\n  Solve:    %.1fs\n  Farfield: %.1fs\n  Total:    %.1fs\n",
                r.t_assembly_s, r.t_solve_s, r.t_farfield_s, total.elapsed_s());
    bem_ctx_destroy(ctx);
    return 0;
}
