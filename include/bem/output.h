// Reference-compatible JSON output (BEM-CPP src/output.h:7-14).
#ifndef BEM_COMPAT_OUTPUT_H
#define BEM_COMPAT_OUTPUT_H

void write_json(const char* filename, const double* M, const double* theta, int ntheta, double ka, double n_re,
                double n_im, int refinements, int n_alpha, int n_beta, int n_gamma, double time_assembly,
                double time_solve, double time_farfield, double time_total);

#endif
