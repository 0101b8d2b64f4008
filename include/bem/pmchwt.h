// Reference-compatible PMCHWT system (BEM-CPP src/pmchwt.h:12-18).
// Z: caller-allocated 2N x 2N row-major; L_ext / K_ext may be NULL.
#ifndef BEM_COMPAT_PMCHWT_H
#define BEM_COMPAT_PMCHWT_H

#include "assembly.h"

void assemble_pmchwt(const RWG& rwg, const Mesh& mesh, std::complex<double> k_ext,
                     std::complex<double> k_int, double eta_ext, double eta_int, int quad_order,
                     std::complex<double>* Z, std::complex<double>* L_ext, std::complex<double>* K_ext);

#endif
