// Reference-compatible dense solver (BEM-CPP src/solver.h:11-22).
// Factors made by lu_factorize_cuda are consumed only by lu_solve_cuda (the
// packed layout is this library's: P Z = L U of the row-major Z).
// Return value: LAPACK-style info (0 = success, k > 0: zero pivot).
#ifndef BEM_COMPAT_SOLVER_H
#define BEM_COMPAT_SOLVER_H

#include <complex>

#include "types.h"

int lu_factorize_cuda(std::complex<double>* Z, int n, int* ipiv);
int lu_solve_cuda(const std::complex<double>* Z, const int* ipiv, int n, std::complex<double>* B, int nrhs);
int lu_solve_full(std::complex<double>* Z, int n, std::complex<double>* B, int nrhs);

#endif
