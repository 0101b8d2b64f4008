// C entry points over the reference's own host-side C++ (mesh.cpp, rwg.cpp,
// rhs.cpp, orient.cpp, graglia.h), compiled from the reference sources in
// place by oracle/Makefile into oracle/_ref/libref_host.so.
//
// TEST INFRASTRUCTURE ONLY: the tests load this library to pin the oracle
// and the product's host code against the reference's own implementation.
#include "mesh.h"
#include "rwg.h"
#include "rhs.h"
#include "orient.h"
#include "graglia.h"
#include "output.h"
#include "quadrature.h"
#include "farfield.h"
#include <cstring>
#include <vector>

static Mesh g_mesh;
static RWG g_rwg;
static std::vector<Orientation> g_or;

// The current mesh and RWG, for the other translation unit of this library
// (ref_asm_shim.cu).
const Mesh& ref_current_mesh() { return g_mesh; }
const RWG& ref_current_rwg() { return g_rwg; }

extern "C" {

// kind 0 = icosphere(radius=param, ref), 1 = hex_prism(aspect=param, ref)
int ref_make_mesh(int kind, double param, int ref, int* nv, int* nt, int* nrwg) {
    g_mesh = (kind == 0) ? icosphere(param, ref) : hex_prism(param, ref);
    g_rwg = build_rwg(g_mesh);
    *nv = g_mesh.nv();
    *nt = g_mesh.nt();
    *nrwg = g_rwg.N;
    return 0;
}

// load_obj (mesh.cpp:156-250) into the current mesh.  No RWG is built (the
// file may hold a non-manifold mesh); the reference reports the removed
// degenerate triangles and the non-manifold edges on stderr only.  The file
// must exist: the reference exits on a missing one.
int ref_load_obj(const char* path, int* nv, int* nt) {
    g_mesh = load_obj(path);
    *nv = g_mesh.nv();
    *nt = g_mesh.nt();
    return 0;
}

// Make (verts, tris) the current mesh (no RWG built).
void ref_set_mesh(const double* verts, int nv, const int* tris, int nt) {
    g_mesh = Mesh();
    for (int i = 0; i < nv; i++) g_mesh.verts.push_back(Vec3(verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]));
    g_mesh.tris.assign(tris, tris + 3 * nt);
}

// Vertex and triangle counts of the current mesh.
void ref_mesh_counts(int* nv, int* nt) {
    *nv = g_mesh.nv();
    *nt = g_mesh.nt();
}

// build_rwg (rwg.cpp:5-43) on the current mesh; fetch with ref_get_rwg.
int ref_build_rwg(void) {
    g_rwg = build_rwg(g_mesh);
    return g_rwg.N;
}

// mesh_volume, mesh_dmax, normalize_mesh (mesh.cpp:252-294) of the current
// mesh; normalize_mesh rescales it in place (fetch it with ref_get_mesh).
double ref_mesh_volume(void) { return mesh_volume(g_mesh); }
double ref_mesh_dmax(void) { return mesh_dmax(g_mesh); }
double ref_normalize_mesh(void) { return normalize_mesh(g_mesh); }

// tri_quadrature (quadrature.h:14-70), unknown orders included.
int ref_tri_quadrature(int order, double* pts, double* wts) {
    TriQuad q = tri_quadrature(order);
    for (int i = 0; i < q.npts; i++) {
        pts[2 * i] = q.pts[i][0];
        pts[2 * i + 1] = q.pts[i][1];
        wts[i] = q.wts[i];
    }
    return q.npts;
}

// write_json (output.cpp:5-64).
void ref_write_json(const char* filename, const double* M, const double* theta, int ntheta, double ka,
                    double n_re, double n_im, int refinements, int na, int nb, int ng, double t_asm,
                    double t_solve, double t_ff, double t_total) {
    write_json(filename, M, theta, ntheta, ka, n_re, n_im, refinements, na, nb, ng, t_asm, t_solve, t_ff,
               t_total);
}

// compute_far_field_vec_batch_cpu (farfield.cu:351-431) on the current mesh
// and RWG: coefficients (N complex each), r_hats (ndir x 3) -> Fv (ndir x 3 complex).
void ref_farfield_cpu(int quad_order, const double* cJ, const double* cM, double k_re, double k_im,
                      double eta_ext, const double* r_hats, int ndir, double* Fv) {
    FFCache cache;
    cache.init(g_rwg, g_mesh, quad_order);
    std::vector<Vec3> rh(ndir);
    for (int d = 0; d < ndir; d++) rh[d] = Vec3(r_hats[3 * d], r_hats[3 * d + 1], r_hats[3 * d + 2]);
    compute_far_field_vec_batch_cpu(cache, reinterpret_cast<const std::complex<double>*>(cJ),
                                    reinterpret_cast<const std::complex<double>*>(cM),
                                    std::complex<double>(k_re, k_im), eta_ext, rh.data(), ndir,
                                    reinterpret_cast<std::complex<double>*>(Fv));
}

// amplitude_to_mueller (farfield.cu:464-508).
void ref_amplitude_to_mueller(const double* S1, const double* S2, const double* S3, const double* S4,
                              int ntheta, double* M) {
    amplitude_to_mueller(reinterpret_cast<const std::complex<double>*>(S1),
                         reinterpret_cast<const std::complex<double>*>(S2),
                         reinterpret_cast<const std::complex<double>*>(S3),
                         reinterpret_cast<const std::complex<double>*>(S4), ntheta, M);
}

int ref_subdivide_flat(void) {
    g_mesh = subdivide_flat(g_mesh);
    g_rwg = build_rwg(g_mesh);
    return g_rwg.N;
}

void ref_get_mesh(double* verts, int* tris) {
    for (int i = 0; i < g_mesh.nv(); i++) {
        verts[3 * i] = g_mesh.verts[i].x;
        verts[3 * i + 1] = g_mesh.verts[i].y;
        verts[3 * i + 2] = g_mesh.verts[i].z;
    }
    std::memcpy(tris, g_mesh.tris.data(), g_mesh.tris.size() * sizeof(int));
}

void ref_get_rwg(int* tri_p, int* tri_m, double* free_p, double* free_m,
                 double* length, double* area_p, double* area_m) {
    for (int n = 0; n < g_rwg.N; n++) {
        tri_p[n] = g_rwg.tri_p[n];
        tri_m[n] = g_rwg.tri_m[n];
        free_p[3 * n] = g_rwg.free_p[n].x; free_p[3 * n + 1] = g_rwg.free_p[n].y; free_p[3 * n + 2] = g_rwg.free_p[n].z;
        free_m[3 * n] = g_rwg.free_m[n].x; free_m[3 * n + 1] = g_rwg.free_m[n].y; free_m[3 * n + 2] = g_rwg.free_m[n].z;
        length[n] = g_rwg.length[n];
        area_p[n] = g_rwg.area_p[n];
        area_m[n] = g_rwg.area_m[n];
    }
}

// b (2N complex as interleaved doubles)
void ref_rhs(double k_re, double k_im, double eta_ext, const double* E0,
             const double* khat, int quad_order, double* b) {
    compute_rhs_planewave(g_rwg, g_mesh, std::complex<double>(k_re, k_im), eta_ext,
                          Vec3(E0[0], E0[1], E0[2]), Vec3(khat[0], khat[1], khat[2]),
                          quad_order, reinterpret_cast<std::complex<double>*>(b));
}

int ref_orientations(int na, int nb, int ng, int bsym, int gsym, int mirror, int sort) {
    g_or = generate_orientations(na, nb, ng, bsym, gsym, mirror != 0);
    if (sort) sort_orientations_nearest(g_or);
    return (int)g_or.size();
}

void ref_get_orientations(double* RT, double* w) {
    for (size_t o = 0; o < g_or.size(); o++) {
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) RT[9 * o + 3 * i + j] = g_or[o].RT.m[i][j];
        w[o] = g_or[o].weight;
    }
}

void ref_graglia(const double* r, const double* v0, const double* v1, const double* v2,
                 int quad_order, double* P, double* V) {
    Vec3 R(r[0], r[1], r[2]), a(v0[0], v0[1], v0[2]), b(v1[0], v1[1], v1[2]), c(v2[0], v2[1], v2[2]);
    TriQuad q = tri_quadrature(quad_order);
    *P = potential_integral_triangle(R, a, b, c);
    Vec3 vv = vector_potential_integral_triangle(R, a, b, c, q);
    V[0] = vv.x; V[1] = vv.y; V[2] = vv.z;
}

}  // extern "C"
