// Reference-compatible operator assembly (BEM-CPP src/assembly.h:11-13).
// L, K: caller-allocated N x N row-major, overwritten.
#ifndef BEM_COMPAT_ASSEMBLY_H
#define BEM_COMPAT_ASSEMBLY_H

#include <complex>

#include "quadrature.h"
#include "rwg.h"

void assemble_L_K_cuda(const RWG& rwg, const Mesh& mesh, std::complex<double> k, int quad_order,
                       std::complex<double>* L, std::complex<double>* K);

#endif
