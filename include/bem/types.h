// Reference-compatible core types for the dense path (the declarations of
// BEM-CPP src/types.h that its dense branch uses): cdouble, Vec3, INV4PI,
// Timer.  Implemented by libbem_compat over libbemdense.
#ifndef BEM_COMPAT_TYPES_H
#define BEM_COMPAT_TYPES_H

#include <chrono>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>

typedef std::complex<double> cdouble;

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
static const double INV4PI = 1.0 / (4.0 * M_PI);

struct Vec3 {
    double x, y, z;
    Vec3() : x(0), y(0), z(0) {}
    Vec3(double a, double b, double c) : x(a), y(b), z(c) {}
    Vec3 operator+(const Vec3& o) const { return Vec3(x + o.x, y + o.y, z + o.z); }
    Vec3 operator-(const Vec3& o) const { return Vec3(x - o.x, y - o.y, z - o.z); }
    Vec3 operator*(double s) const { return Vec3(x * s, y * s, z * s); }
    double dot(const Vec3& o) const { return x * o.x + y * o.y + z * o.z; }
    Vec3 cross(const Vec3& o) const { return Vec3(y * o.z - z * o.y, z * o.x - x * o.z, x * o.y - y * o.x); }
    double norm() const { return std::sqrt(x * x + y * y + z * z); }
    double norm2() const { return x * x + y * y + z * z; }
    Vec3 normalized() const {
        double n = norm();
        return Vec3(x / n, y / n, z / n);
    }
};
inline Vec3 operator*(double s, const Vec3& v) { return v * s; }

struct Timer {
    std::chrono::high_resolution_clock::time_point t0;
    Timer() { reset(); }
    void reset() { t0 = std::chrono::high_resolution_clock::now(); }
    double elapsed_ms() const {
        return std::chrono::duration<double, std::milli>(std::chrono::high_resolution_clock::now() - t0).count();
    }
    double elapsed_s() const { return elapsed_ms() / 1000.0; }
};

#endif
