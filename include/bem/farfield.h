// Reference-compatible far field / Mueller interface (BEM-CPP
// src/farfield.h:9-71).  FFCacheGPU owns a device-resident geometry.
#ifndef BEM_COMPAT_FARFIELD_H
#define BEM_COMPAT_FARFIELD_H

#include <complex>
#include <vector>

#include "rwg.h"

struct FFCache {
    std::vector<double> qpts;   // (2 N Nq, 3)
    std::vector<double> fvals;  // (2 N Nq, 3)
    std::vector<double> jw;     // (2 N Nq)
    int N, Nq;
    // mesh kept for the device upload
    std::vector<double> mesh_verts;
    std::vector<int> mesh_tris;
    int quad_order;
    void init(const RWG& rwg, const Mesh& mesh, int quad_order);
};

struct FFCacheGPU {
    double* d_qpts;
    double* d_fvals;
    double* d_jw;
    int N, Nq;
    bool initialized;
    void* geom;  // bem_geom*
    FFCacheGPU() : d_qpts(0), d_fvals(0), d_jw(0), N(0), Nq(0), initialized(false), geom(0) {}
    void upload(const FFCache& cache);
    void free();
    ~FFCacheGPU();
};

void compute_farfield_batch_cuda(const FFCacheGPU& gpu_cache, const std::complex<double>* coeffs_J,
                                 const std::complex<double>* coeffs_M, const double* r_hats,
                                 std::complex<double> k_ext, double eta_ext, int n_calls, int n_orient, int ndir,
                                 std::complex<double>* Fv_out);

void compute_far_field_vec_batch_cpu(const FFCache& cache, const std::complex<double>* coeffs_J,
                                     const std::complex<double>* coeffs_M, std::complex<double> k_ext,
                                     double eta_ext, const Vec3* r_hats, int ndir, std::complex<double>* Fv_out);

void compute_far_field(const FFCache& cache, const std::complex<double>* coeffs_J,
                       const std::complex<double>* coeffs_M, std::complex<double> k_ext, double eta_ext,
                       const double* theta_arr, int ntheta, std::complex<double>* F_theta,
                       std::complex<double>* F_phi);

void amplitude_to_mueller(const std::complex<double>* S1, const std::complex<double>* S2,
                          const std::complex<double>* S3, const std::complex<double>* S4, int ntheta, double* M);

#endif
