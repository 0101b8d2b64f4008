// Device helpers shared by the assembly kernels (assembly.cu) and the
// shape-gradient kernels (grad_geom.cu): complex arithmetic, the Green's
// function pieces and the Graglia singular integrals.
#pragma once
#include <cuda_runtime.h>

#include <cmath>

namespace bem {

#define INV4PI_D 0.079577471545947667884

// ------------------------------------------------------------ complex helpers
struct cplx {
    double re, im;
};
__device__ __forceinline__ cplx cmul(cplx a, cplx b) {
    return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}

struct Medium {
    double kr, ki;  // k = kr + i ki
};

// e^-x for x >= 0.  Below 2^-54 the correctly rounded value is exactly 1;
// the literal G_smooth at coincident points (R_s = 1e-15) subtracts
// 1/(4 pi R_s) from e^-x cos(k R_s)/(4 pi R_s), so one unit in the last
// place of e^-x there would become 0.0156 in G.
__device__ __forceinline__ double exp_decay(double x) { return x < 5.551115123125783e-17 ? 1.0 : exp(-x); }

// G_smooth = (exp(ikR) - 1)/(4 pi R) without cancellation (limit ik/(4 pi)).
__device__ __forceinline__ cplx g_smooth_exact(Medium k, double R) {
    if (R == 0.0) return {-k.ki * INV4PI_D, k.kr * INV4PI_D};
    double s, c, sh, ch;
    sincos(k.kr * R, &s, &c);
    sincos(0.5 * k.kr * R, &sh, &ch);
    double re = expm1(-k.ki * R) * c - 2.0 * sh * sh;
    double im = exp(-k.ki * R) * s;
    double f = INV4PI_D / R;
    return {re * f, im * f};
}

// ------------------------------------------------------------ Graglia (FP64)
struct TriQ {
    int n;
    double l1[25], l2[25], w[25];
};

// int_T 1/|r - r'| dS' (Graglia 1993) -- graglia.h:11-66, same guards.
__device__ inline double potential_integral(double rx, double ry, double rz, const double* v) {
    const double ax = v[0], ay = v[1], az = v[2], bx = v[3], by = v[4], bz = v[5],
                 cx = v[6], cy = v[7], cz = v[8];
    double e1x = bx - ax, e1y = by - ay, e1z = bz - az;
    double e2x = cx - ax, e2y = cy - ay, e2z = cz - az;
    double nx = e1y * e2z - e1z * e2y, ny = e1z * e2x - e1x * e2z, nz = e1x * e2y - e1y * e2x;
    double nn = sqrt(nx * nx + ny * ny + nz * nz);
    if (nn < 1e-15) return 0.0;
    nx /= nn, ny /= nn, nz /= nn;
    double res = 0.0;
    for (int i = 0; i < 3; i++) {
        const double* vi = v + 3 * i;
        const double* vj = v + 3 * ((i + 1) % 3);
        double ex = vj[0] - vi[0], ey = vj[1] - vi[1], ez = vj[2] - vi[2];
        double le = sqrt(ex * ex + ey * ey + ez * ez);
        if (le < 1e-15) continue;
        double tx = ex / le, ty = ey / le, tz = ez / le;
        double mx = ny * tz - nz * ty, my = nz * tx - nx * tz, mz = nx * ty - ny * tx;
        double dix = rx - vi[0], diy = ry - vi[1], diz = rz - vi[2];
        double d = dix * mx + diy * my + diz * mz;
        double h = dix * nx + diy * ny + diz * nz;
        double djx = vj[0] - rx, djy = vj[1] - ry, djz = vj[2] - rz;
        double dkx = vi[0] - rx, dky = vi[1] - ry, dkz = vi[2] - rz;
        double sp = djx * tx + djy * ty + djz * tz;
        double sm = dkx * tx + dky * ty + dkz * tz;
        double Rp = sqrt(djx * djx + djy * djy + djz * djz);
        double Rm = sqrt(dkx * dkx + dky * dky + dkz * dkz);
        if (Rp + sp > 1e-15 && Rm + sm > 1e-15) {
            double arg = (Rp + sp) / (Rm + sm);
            if (arg > 0) res += d * log(arg);
        }
        double ah = fabs(h);
        if (ah > 1e-15) {
            double R0 = d * d + h * h;
            double t1 = atan2(d * sp, R0 + ah * Rp);
            double t2 = atan2(d * sm, R0 + ah * Rm);
            res -= ah * (t1 - t2);
        }
    }
    return res;
}

// int_T |r - r'| dS' by the triangle rule -- graglia.h:69-85.  Evaluated with
// explicitly rounded operations (no FMA contraction) in the reference's
// order: the central difference below divides by 2e-6, so W must round the
// way the reference rounds it.
__device__ inline double integral_R(double rx, double ry, double rz, const double* v, const TriQ& q) {
    double e1x = __dsub_rn(v[3], v[0]), e1y = __dsub_rn(v[4], v[1]), e1z = __dsub_rn(v[5], v[2]);
    double e2x = __dsub_rn(v[6], v[0]), e2y = __dsub_rn(v[7], v[1]), e2z = __dsub_rn(v[8], v[2]);
    double nx = __dsub_rn(__dmul_rn(e1y, e2z), __dmul_rn(e1z, e2y));
    double ny = __dsub_rn(__dmul_rn(e1z, e2x), __dmul_rn(e1x, e2z));
    double nz = __dsub_rn(__dmul_rn(e1x, e2y), __dmul_rn(e1y, e2x));
    double area = __dmul_rn(0.5, __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(nx, nx), __dmul_rn(ny, ny)),
                                                      __dmul_rn(nz, nz))));
    double acc = 0.0;
    for (int k = 0; k < q.n; k++) {
        double l0 = __dsub_rn(__dsub_rn(1.0, q.l1[k]), q.l2[k]);
        double px = __dadd_rn(__dadd_rn(__dmul_rn(l0, v[0]), __dmul_rn(q.l1[k], v[3])), __dmul_rn(q.l2[k], v[6]));
        double py = __dadd_rn(__dadd_rn(__dmul_rn(l0, v[1]), __dmul_rn(q.l1[k], v[4])), __dmul_rn(q.l2[k], v[7]));
        double pz = __dadd_rn(__dadd_rn(__dmul_rn(l0, v[2]), __dmul_rn(q.l1[k], v[5])), __dmul_rn(q.l2[k], v[8]));
        double dx = __dsub_rn(px, rx), dy = __dsub_rn(py, ry), dz = __dsub_rn(pz, rz);
        double R = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
        acc = __dadd_rn(acc, __dmul_rn(q.w[k], R));
    }
    return __dmul_rn(area, acc);
}

// P = int_T 1/|r - r'| dS' and V = r P - grad_r W (W = int_T |r - r'| dS',
// central differences with eps = 1e-6) at the point of barycentric
// coordinates (l1, l2) of triangle v -- graglia.h:90-112.
__device__ inline void graglia_point(const double* v, double l1, double l2, const TriQ& q, double* P, double* V) {
    double l0 = __dsub_rn(__dsub_rn(1.0, l1), l2);
    double r[3];
    for (int d = 0; d < 3; d++)
        r[d] = __dadd_rn(__dadd_rn(__dmul_rn(v[d], l0), __dmul_rn(v[3 + d], l1)), __dmul_rn(v[6 + d], l2));
    double p = potential_integral(r[0], r[1], r[2], v);
    const double eps = 1e-6;
    double g[3];
    for (int d = 0; d < 3; d++) {
        double rp[3] = {r[0], r[1], r[2]}, rm[3] = {r[0], r[1], r[2]};
        rp[d] = __dadd_rn(rp[d], eps);
        rm[d] = __dsub_rn(rm[d], eps);
        double wp = integral_R(rp[0], rp[1], rp[2], v, q);
        double wm = integral_R(rm[0], rm[1], rm[2], v, q);
        g[d] = __ddiv_rn(__dsub_rn(wp, wm), 2.0 * eps);
    }
    *P = p;
    for (int d = 0; d < 3; d++) V[d] = __dsub_rn(__dmul_rn(r[d], p), g[d]);
}

}  // namespace bem
