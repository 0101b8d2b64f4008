// Reference-compatible plane-wave excitation (BEM-CPP src/rhs.h:11-15).
#ifndef BEM_COMPAT_RHS_H
#define BEM_COMPAT_RHS_H

#include <complex>

#include "rwg.h"

void compute_rhs_planewave(const RWG& rwg, const Mesh& mesh, std::complex<double> k_ext, double eta_ext,
                           const Vec3& E0, const Vec3& k_hat, int quad_order, std::complex<double>* b);

#endif
