// Context: device, stream, error reporting, workspace.
#include <cstdarg>
#include <cstring>

#include "bem_internal.h"

namespace bem {

int fail(bem_ctx* ctx, int status, const char* fmt, ...) {
    if (ctx) {
        char buf[1024];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        ctx->last_error = buf;
    }
    return status;
}

}  // namespace bem

int bem_ctx::ensure_ws(size_t bytes) {
    if (bytes <= ws_bytes) return BEM_OK;
    if (ws) cudaFree(ws);
    ws = nullptr;
    ws_bytes = 0;
    cudaError_t e = cudaMalloc(&ws, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return bem::fail(this, BEM_ERR_OOM, "workspace of %zu bytes: %s", bytes,
                         cudaGetErrorString(e));
    }
    ws_bytes = bytes;
    return BEM_OK;
}

extern "C" {

const char* bem_version(void) { return "bem-b200 0.1 (sm_100a)"; }

int bem_ctx_create(int device, bem_ctx** out) {
    if (!out) return BEM_ERR_INVALID;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return BEM_ERR_NODEVICE;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10) {
        cudaGetLastError();
        return BEM_ERR_NODEVICE;
    }
    bem_ctx* c = new bem_ctx();
    c->device = device;
    c->sm_count = prop.multiProcessorCount;
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&c->d_status, 64 * sizeof(int)) != cudaSuccess ||
        cudaMemset(c->d_status, 0, 64 * sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        delete c;
        return BEM_ERR_CUDA;
    }
    c->stream = c->own_stream;
    *out = c;
    return BEM_OK;
}

int bem_ctx_destroy(bem_ctx* ctx) {
    if (!ctx) return BEM_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    if (ctx->ws) cudaFree(ctx->ws);
    if (ctx->d_status) cudaFree(ctx->d_status);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return BEM_OK;
}

int bem_ctx_set_stream(bem_ctx* ctx, void* stream) {
    if (!ctx) return BEM_ERR_INVALID;
    // NULL selects the legacy default stream (what torch's default stream is)
    ctx->stream = (cudaStream_t)stream;
    return BEM_OK;
}

int bem_ctx_synchronize(bem_ctx* ctx) {
    if (!ctx) return BEM_ERR_INVALID;
    BEM_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return BEM_OK;
}

const char* bem_last_error(const bem_ctx* ctx) { return ctx ? ctx->last_error.c_str() : ""; }

int64_t bem_ctx_launch_count(const bem_ctx* ctx) { return ctx ? ctx->launches : 0; }

}  // extern "C"
