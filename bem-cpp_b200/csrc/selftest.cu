// The failure path of a bounded device-side wait, exercised without a fault.
//
// Every wait in this library's kernels (the tensor-core pipelines' mbarriers,
// the int8 residual's pacing) gives up after a fixed number of SM clock
// cycles, records BEM_ERR_TIMEOUT in a status word and returns, so a stuck
// producer surfaces as an error status while the context stays usable.  This
// entry point runs that pattern alone: one thread waits on a device flag for
// at most `cycles` clock cycles.  With the flag left at 0 nothing ever sets it
// and the wait runs out; with the flag set the wait ends at once.
#include <cuda_runtime.h>

#include <cstdint>

#include "bem_internal.h"

namespace bem {
namespace {

__global__ void bounded_wait_kernel(const volatile int* flag, long long cycles, int* status) {
    const long long t0 = clock64();
    while (*flag == 0) {
        if (clock64() - t0 > cycles) {
            *status = (int)BEM_ERR_TIMEOUT;
            return;
        }
    }
    *status = (int)BEM_OK;
}

}  // namespace
}  // namespace bem

extern "C" int bem_selftest_bounded_wait(bem_ctx* ctx, int64_t cycles, int set_flag) {
    if (!ctx || cycles < 0 || cycles > 4000000000LL) return BEM_ERR_INVALID;
    BEM_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    int* d = nullptr;
    BEM_TRY_CUDA(ctx, cudaMalloc(&d, 2 * sizeof(int)));
    const int h[2] = {set_flag ? 1 : 0, -1};  // flag, status
    int st = -1;
    cudaError_t e = cudaMemcpyAsync(d, h, sizeof(h), cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) {
        bem::bounded_wait_kernel<<<1, 1, 0, ctx->stream>>>(d, (long long)cycles, d + 1);
        ctx->launches++;
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&st, d + 1, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(d);
    if (e != cudaSuccess) return bem::fail(ctx, BEM_ERR_CUDA, "bounded wait: %s", cudaGetErrorString(e));
    if (st == BEM_ERR_TIMEOUT)
        return bem::fail(ctx, BEM_ERR_TIMEOUT, "bounded wait ran out after %lld clock cycles", (long long)cycles);
    if (st != BEM_OK) return bem::fail(ctx, BEM_ERR_CUDA, "bounded wait: status %d", st);
    return BEM_OK;
}
