// 3xTF32 complex GEMM on the fifth-generation tensor cores (tcgen05).
// (placeholder: hooks disabled until the tensor-core kernel lands)
#include "lu_internal.h"

namespace bem {
TrailingUpdate<float> tc_update_fp32(bem_ctx*) { return TrailingUpdate<float>(); }
}  // namespace bem
