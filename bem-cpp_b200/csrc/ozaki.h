// Int8 tensor-core (Ozaki scheme) FP64 residual: shared declarations.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "bem_internal.h"

namespace bem {
namespace oz {
constexpr int S_MAX = 8;  // largest digit count supported
}

// Digit planes of the fixed matrix Z' (made once per factorisation).
struct OzakiZ {
    int n = 0, S = 0;
    int64_t ldk = 0;    // bytes per digit row (2n rounded up to 128)
    int64_t plane = 0;  // bytes per digit plane (n * ldk)
    int8_t* A = nullptr;
    int* e = nullptr;   // per-row power-of-two exponents
    int device = -1;    // where A and e live
    const void* owner = nullptr;  // context whose stream uses them
};

size_t ozaki_z_bytes(int n, int S);
int ozaki_prepare_z(bem_ctx* ctx, OzakiZ* oz, const double2* Z, int64_t ldz, int n, int S);
void ozaki_free(OzakiZ* oz);
// R -= Z X with FP64 accuracy (R holds B on entry).  x_digits > 0 (with
// round_x): X is first rounded in place to its first x_digits digits (7 bits
// each below its column's exponent), and R -= Z X is exact for the rounded X
// up to the truncation of Z's digits; the digit pairs of the dropped X digits
// are not computed.
int ozaki_residual(bem_ctx* ctx, const OzakiZ* oz, const double2* X, int64_t ldx, double2* R, int64_t ldr,
                   int nrhs, int x_digits = 0, double2* round_x = nullptr);
// R -= Z (scale[j] D[:, j]) with `digits` (<= oz->S) digits: the update form
// r_{k+1} = r_k - Z d_k of the refinement residual.  d_digits > 0 (with
// fix_x): d is rounded to its first d_digits digits and the iterate fix_x,
// which already holds x_k + d, is corrected to x_k + (rounded d).
int ozaki_residual_update(bem_ctx* ctx, const OzakiZ* oz, const float2* D, int64_t ldd, const double* scale,
                          double2* R, int64_t ldr, int nrhs, int digits, int d_digits = 0, double2* fix_x = nullptr,
                          int64_t ldfix = 0);
}  // namespace bem
