// Context: device, stream, error reporting, workspace.
#include <cstdarg>
#include <cstring>
#include <mutex>
#include <set>

#include "bem_internal.h"
#include "ozaki.h"

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

int h2d(bem_ctx* ctx, void* dst, const void* src, size_t bytes) {
    if (bytes == 0) return BEM_OK;
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
    return BEM_OK;
}

int d2h(bem_ctx* ctx, void* dst, const void* src, size_t bytes) {
    if (bytes == 0) return BEM_OK;
    BEM_TRY_CUDA(ctx, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    BEM_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return BEM_OK;
}

}  // namespace bem

cudaEvent_t bem_ctx::prof_begin(int cls) {
    (void)cls;
    if (!prof) return nullptr;
    cudaEvent_t e;
    if (!prof_pool.empty()) {
        e = prof_pool.back();
        prof_pool.pop_back();
    } else if (cudaEventCreate(&e) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    cudaEventRecord(e, stream);
    return e;
}

void bem_ctx::prof_end(int cls, cudaEvent_t a, double flops, double bytes) {
    if (!prof || !a) return;
    cudaEvent_t b;
    if (!prof_pool.empty()) {
        b = prof_pool.back();
        prof_pool.pop_back();
    } else if (cudaEventCreate(&b) != cudaSuccess) {
        cudaGetLastError();
        prof_pool.push_back(a);
        return;
    }
    cudaEventRecord(b, stream);
    prof_pending.push_back({cls, a, b, flops, bytes});
    if (prof_pending.size() > 65536) prof_collect();  // (collecting synchronizes the stream)
}

int bem_ctx::prof_collect() {
    if (prof_pending.empty()) return BEM_OK;
    if (cudaStreamSynchronize(stream) != cudaSuccess) return BEM_ERR_CUDA;
    for (auto& p : prof_pending) {
        float ms = 0;
        cudaEventElapsedTime(&ms, p.a, p.b);
        prof_launches[p.cls]++;
        prof_ms[p.cls] += ms;
        prof_flops[p.cls] += p.flops;
        prof_bytes[p.cls] += p.bytes;
        prof_pool.push_back(p.a);
        prof_pool.push_back(p.b);
    }
    prof_pending.clear();
    return BEM_OK;
}

namespace bem {
namespace {
struct CachedBlock {
    void* p;
    size_t bytes;
    const void* owner;  // context whose stream last used the block (null: synchronised)
};
struct DevCache {
    bool on = false;
    std::vector<CachedBlock> blocks;
};
std::mutex g_cache_mu;
DevCache g_cache[64];
std::set<const void*> g_owners;  // live contexts

void free_blocks_locked(int device, const void* owner, bool all) {
    DevCache& c = g_cache[device];
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    for (size_t i = 0; i < c.blocks.size();) {
        if (all || c.blocks[i].owner == owner) {
            cudaFree(c.blocks[i].p);
            c.blocks.erase(c.blocks.begin() + i);
        } else {
            i++;
        }
    }
    cudaSetDevice(prev);
}
}  // namespace

void devmem_owner(const void* owner, bool alive) {
    std::lock_guard<std::mutex> g(g_cache_mu);
    if (alive) {
        g_owners.insert(owner);
        return;
    }
    g_owners.erase(owner);
    for (int d = 0; d < 64; d++)
        if (!g_cache[d].blocks.empty()) free_blocks_locked(d, owner, false);
}

void* devmem_alloc(int device, size_t bytes, const void* owner) {
    if (device >= 0 && device < 64) {
        std::lock_guard<std::mutex> g(g_cache_mu);
        auto& bl = g_cache[device].blocks;
        for (size_t i = 0; i < bl.size(); i++)
            if (bl[i].bytes == bytes && (bl[i].owner == owner || bl[i].owner == nullptr)) {
                void* p = bl[i].p;
                bl.erase(bl.begin() + i);
                return p;
            }
    }
    void* p = nullptr;
    if (cudaMalloc(&p, bytes) == cudaSuccess) return p;
    cudaGetLastError();
    if (device < 0 || device >= 64) return nullptr;
    {
        std::lock_guard<std::mutex> g(g_cache_mu);
        if (g_cache[device].blocks.empty()) return nullptr;
        free_blocks_locked(device, nullptr, true);
    }
    if (cudaMalloc(&p, bytes) == cudaSuccess) return p;
    cudaGetLastError();
    return nullptr;
}

void devmem_free(int device, void* p, size_t bytes, const void* owner) {
    if (!p) return;
    if (device >= 0 && device < 64) {
        std::lock_guard<std::mutex> g(g_cache_mu);
        if (g_cache[device].on) {
            // a block goes back to the live context that used it: its next
            // user is that context's stream, ordered after the work still
            // reading it.  Without a live owner, wait for the device first.
            if (!owner || !g_owners.count(owner)) {
                int prev = 0;
                cudaGetDevice(&prev);
                cudaSetDevice(device);
                cudaDeviceSynchronize();
                cudaSetDevice(prev);
                owner = nullptr;
            }
            g_cache[device].blocks.push_back({p, bytes, owner});
            return;
        }
    }
    cudaFree(p);
}

bool devmem_cache_enabled(int device) {
    if (device < 0 || device >= 64) return false;
    std::lock_guard<std::mutex> g(g_cache_mu);
    return g_cache[device].on;
}

void devmem_cache_enable(int device, bool on) {
    if (device < 0 || device >= 64) return;
    std::lock_guard<std::mutex> g(g_cache_mu);
    g_cache[device].on = on;
    if (!on && !g_cache[device].blocks.empty()) free_blocks_locked(device, nullptr, true);
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
    bem::devmem_owner(c, true);
    *out = c;
    return BEM_OK;
}

int bem_ctx_destroy(bem_ctx* ctx) {
    if (!ctx) return BEM_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    bem::devmem_owner(ctx, false);  // frees the cached blocks it owns
    if (ctx->ws) cudaFree(ctx->ws);
    if (ctx->tc_buf) cudaFree(ctx->tc_buf);
    if (ctx->oz_buf) cudaFree(ctx->oz_buf);
    if (ctx->d_status) cudaFree(ctx->d_status);
    for (auto& p : ctx->prof_pending) cudaEventDestroy(p.a), cudaEventDestroy(p.b);
    for (auto e : ctx->prof_pool) cudaEventDestroy(e);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return BEM_OK;
}

int bem_ctx_set_stream(bem_ctx* ctx, void* stream) {
    if (!ctx) return BEM_ERR_INVALID;
    // NULL selects the legacy default stream (what torch's default stream is).
    // Cached blocks of this context are reused in stream order: finish the
    // old stream's work first.
    cudaStreamSynchronize(ctx->stream);
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

int bem_ctx_set_option(bem_ctx* ctx, const char* name, int value) {
    if (!ctx || !name) return BEM_ERR_INVALID;
    if (!std::strcmp(name, "residual_pace_epoch")) {
        if (value < 0) return bem::fail(ctx, BEM_ERR_INVALID, "residual_pace_epoch must be >= 0");
        ctx->oz_pace_epoch = value;
    } else if (!std::strcmp(name, "residual_pace_lead")) {
        if (value < 0) return bem::fail(ctx, BEM_ERR_INVALID, "residual_pace_lead must be >= 0");
        ctx->oz_pace_lead = value;
    } else if (!std::strcmp(name, "panel_clusters")) {
        ctx->panel_clusters = value != 0;
    } else if (!std::strcmp(name, "gmres_digits")) {
        if (value != 0 && (value < 2 || value > bem::oz::S_MAX))
            return bem::fail(ctx, BEM_ERR_INVALID, "gmres_digits must be 0 or 2..%d", bem::oz::S_MAX);
        ctx->gmres_digits = value;
    } else if (!std::strcmp(name, "factor_superblock") || !std::strcmp(name, "solve_superblock")) {
        if (value < 1 || value > 4) return bem::fail(ctx, BEM_ERR_INVALID, "%s must be 1..4", name);
        (name[0] == 'f' ? ctx->factor_sb : ctx->solve_sb) = value;
    } else if (!std::strcmp(name, "cache_factor_memory")) {
        bem::devmem_cache_enable(ctx->device, value != 0);
    } else if (!std::strcmp(name, "farfield_kernel")) {
        if (value != 0 && value != 1) return bem::fail(ctx, BEM_ERR_INVALID, "farfield_kernel must be 0 or 1");
        ctx->ff_kernel = value;
    } else if (!std::strcmp(name, "assembly_kernel")) {
        if (value != 0 && value != 1) return bem::fail(ctx, BEM_ERR_INVALID, "assembly_kernel must be 0 or 1");
        ctx->asm_kernel = value;
    } else if (!std::strcmp(name, "gemm_group_m")) {
        if (value < 1 || value > 512) return bem::fail(ctx, BEM_ERR_INVALID, "gemm_group_m must be 1..512");
        ctx->tc_group_m = value;
    } else if (!std::strcmp(name, "persistent_gemm")) {
        ctx->tc_persistent = value != 0;
    } else if (!std::strcmp(name, "residual_x_digits")) {
        if (value < 0 || value > 7) return bem::fail(ctx, BEM_ERR_INVALID, "residual_x_digits must be 0..7");
        ctx->oz_xdigits = value;
    } else if (!std::strcmp(name, "lu_u12_slabs")) {
        ctx->lu_u12_slabs = value != 0;
    } else if (!std::strcmp(name, "solve_block_inverse")) {
        ctx->solve_inv = value != 0;
    } else if (!std::strcmp(name, "ldlt_cluster_diag")) {
        ctx->ldlt_cluster = value != 0;
    } else if (!std::strcmp(name, "fp64_gemm_3m")) {
        ctx->dmma_3m = value != 0;
    } else if (!std::strcmp(name, "gemm_pairs")) {
        ctx->tc_pair = value != 0;
    } else if (!std::strcmp(name, "batch_buckets")) {
        ctx->batch_buckets = value != 0;
    } else if (!std::strcmp(name, "lu_autotune")) {
        ctx->lu_autotune = value != 0;
    } else if (!std::strcmp(name, "gradient_method")) {
        if (value != 0 && value != 1) return bem::fail(ctx, BEM_ERR_INVALID, "gradient_method must be 0 or 1");
        ctx->grad_method = value;
    } else if (!std::strcmp(name, "verify_columns")) {
        if (value < -1) return bem::fail(ctx, BEM_ERR_INVALID, "verify_columns must be -1, 0 or a column count");
        ctx->verify_cols = value;
    } else if (!std::strcmp(name, "tensor_split")) {
        if (value != 0 && value != 1) return bem::fail(ctx, BEM_ERR_INVALID, "tensor_split must be 0 or 1");
        ctx->tc_split = value;
    } else {
        return bem::fail(ctx, BEM_ERR_INVALID, "unknown option '%s'", name);
    }
    return BEM_OK;
}

int bem_ctx_set_symmetric(bem_ctx* ctx, int mode) {
    if (!ctx) return BEM_ERR_INVALID;
    if (mode != 0 && mode != 1) return bem::fail(ctx, BEM_ERR_INVALID, "symmetric mode must be 0 or 1");
    ctx->sym_mode = mode;
    return BEM_OK;
}

int bem_ctx_set_residual_digits(bem_ctx* ctx, int digits) {
    if (!ctx) return BEM_ERR_INVALID;
    if (digits != 0 && (digits < 2 || digits > bem::oz::S_MAX))
        return bem::fail(ctx, BEM_ERR_INVALID, "residual digits must be 0 or 2..%d", bem::oz::S_MAX);
    ctx->oz_digits = digits;
    return BEM_OK;
}

int bem_ctx_set_tensor_cores(bem_ctx* ctx, int enable) {
    if (!ctx) return BEM_ERR_INVALID;
    ctx->use_tc = enable != 0;
    return BEM_OK;
}

int bem_ctx_profile(bem_ctx* ctx, int enable) {
    if (!ctx) return BEM_ERR_INVALID;
    int s = ctx->prof_collect();
    if (enable) {
        for (int i = 0; i < PROF_NCLASS; i++)
            ctx->prof_launches[i] = 0, ctx->prof_ms[i] = ctx->prof_flops[i] = ctx->prof_bytes[i] = 0;
    }
    ctx->prof = enable != 0;
    return s;
}

int bem_ctx_profile_read(bem_ctx* ctx, int cls, int64_t* launches, double* ms, double* flops,
                         double* bytes) {
    if (!ctx || cls < 0 || cls >= PROF_NCLASS) return BEM_ERR_INVALID;
    int s = ctx->prof_collect();
    if (launches) *launches = ctx->prof_launches[cls];
    if (ms) *ms = ctx->prof_ms[cls];
    if (flops) *flops = ctx->prof_flops[cls];
    if (bytes) *bytes = ctx->prof_bytes[cls];
    return s;
}

}  // extern "C"
