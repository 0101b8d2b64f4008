// Reference-compatible triangle quadrature (BEM-CPP src/quadrature.h:9-14):
// Dunavant rules of orders 4, 7, 13 (other orders give the 7-point rule).
#ifndef BEM_COMPAT_QUADRATURE_H
#define BEM_COMPAT_QUADRATURE_H

#include "../bem_dense.h"

struct TriQuad {
    int npts;
    double pts[25][2];  // (lambda1, lambda2)
    double wts[25];     // sum to 1
};

inline TriQuad tri_quadrature(int order) {
    TriQuad q;
    double p[50], w[25];
    int n = 0;
    if (bem_tri_quadrature(order, &n, p, w) != BEM_OK) bem_tri_quadrature(7, &n, p, w);
    q.npts = n;
    for (int i = 0; i < n; i++) {
        q.pts[i][0] = p[2 * i];
        q.pts[i][1] = p[2 * i + 1];
        q.wts[i] = w[i];
    }
    return q;
}

#endif
