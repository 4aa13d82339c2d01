// mc_context.cu - contexts, error reporting, device buffers, environment maps.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "mc_internal.h"

namespace {
thread_local char g_last_error[512] = "";

// Alias tables of the environment maps made by mc_env_create, keyed by the
// map's col_cdf pointer (the table lives in the same allocation, after it).
std::mutex g_alias_mutex;
std::unordered_map<const void*, const void*> g_alias_tables;
}

namespace mc {

mc_status set_error(mc_status s, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
    return s;
}

mc_status cuda_error(int err, const char* what, const char* file, int line) {
    cudaError_t e = (cudaError_t)err;
    mc_status s = (e == cudaErrorMemoryAllocation) ? MC_ERR_OOM : MC_ERR_CUDA;
    const char* base = std::strrchr(file, '/');
    return set_error(s, "%s failed at %s:%d: %s", what, base ? base + 1 : file, line, cudaGetErrorString(e));
}

mc_status status_from_device_flags(int flags) {
    if (flags == 0) return MC_OK;
    if (flags & MC_DEVERR_TIMEOUT) return set_error(MC_ERR_TIMEOUT, "a bounded device wait ran out (flags 0x%x)", flags);
    if (flags & MC_DEVERR_STACK) return set_error(MC_ERR_STACK_OVERFLOW, "a traversal stack would have overflowed (flags 0x%x)", flags);
    if (flags & MC_DEVERR_QUEUE) return set_error(MC_ERR_QUEUE_OVERFLOW, "a queue append went past its capacity (flags 0x%x)", flags);
    return set_error(MC_ERR_INVALID, "invalid input seen on the device (flags 0x%x)", flags);
}

mc_status devbuf_reserve(DevBuf& b, size_t bytes) {
    if (bytes <= b.bytes && b.ptr) return MC_OK;
    if (b.ptr) cudaFree(b.ptr);
    b.ptr = nullptr;
    b.bytes = 0;
    size_t want = bytes < 256 ? 256 : bytes;
    cudaError_t e = cudaMalloc(&b.ptr, want);
    if (e != cudaSuccess) {
        cudaGetLastError();
        b.ptr = nullptr;
        return set_error(MC_ERR_OOM, "device allocation of %zu bytes failed: %s", want, cudaGetErrorString(e));
    }
    b.bytes = want;
    return MC_OK;
}

void devbuf_free(DevBuf& b) {
    if (b.ptr) cudaFree(b.ptr);
    b.ptr = nullptr;
    b.bytes = 0;
}

// One stream-ordered memory pool per device for the BVH build's buffers. It
// keeps what is freed (release threshold: never), so a build after the first
// takes its memory without a driver allocation; plain cudaMalloc / cudaFree
// pairs per build cost from well under a millisecond to hundreds of
// milliseconds each. The pools live as long as the process: a tree may
// outlive the context that built it.
namespace {
std::mutex g_pool_mutex;
std::unordered_map<int, cudaMemPool_t> g_pools;
}

static cudaMemPool_t device_pool(int device) {
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    auto it = g_pools.find(device);
    if (it != g_pools.end()) return it->second;
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    unsigned long long keep = ~0ull;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    g_pools[device] = pool;
    return pool;
}

mc_status pool_alloc(mc_context* ctx, void** p, size_t bytes) {
    *p = nullptr;
    cudaMemPool_t pool = device_pool(ctx->device);
    if (!pool) return set_error(MC_ERR_CUDA, "device %d: memory pool creation failed", ctx->device);
    cudaError_t e = cudaMallocFromPoolAsync(p, bytes < 256 ? 256 : bytes, pool, ctx->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return set_error(MC_ERR_OOM, "device allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
    }
    return MC_OK;
}

void pool_free(mc_context* ctx, void* p) {
    if (p) cudaFreeAsync(p, ctx->stream);
}

// For a caller that has made the pool's device current and waited for the
// work that reads p.
void pool_release(void* p) {
    if (p) cudaFreeAsync(p, 0);
}

void pool_trim(int device) {
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    auto it = g_pools.find(device);
    if (it != g_pools.end()) cudaMemPoolTrimTo(it->second, 0);
}

// One lane polls *flag (system-scope acquire loads, so a flag in mapped host
// memory or a peer's memory is seen) with a back-off sleep, until it reaches
// value or the device clock says timeout_ns have passed; then the error word
// records the time-out and the stream moves on. Nothing else waits on this
// kernel's lanes, and it touches no other memory.
__global__ void k_wait_value(const uint32_t* flag, uint32_t value, long long timeout_ns, int* err) {
    if (threadIdx.x != 0) return;
    unsigned long long t0, now;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    unsigned sleep = 32;
    // the clock bounds the wait; the iteration count bounds it too, should
    // the clock not advance
    const long long maxIter = (timeout_ns >> 5) + (1ll << 20);
    for (long long it = 0; it < maxIter; it++) {
        uint32_t v;
        asm volatile("ld.acquire.sys.global.u32 %0, [%1];" : "=r"(v) : "l"(flag) : "memory");
        if (v >= value) return;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
        if ((long long)(now - t0) > timeout_ns) {
            atomicOr(err, MC_DEVERR_TIMEOUT);
            return;
        }
        __nanosleep(sleep);
        if (sleep < 4096) sleep <<= 1;
    }
    atomicOr(err, MC_DEVERR_TIMEOUT);
}

}  // namespace mc

extern "C" {

const char* mc_version(void) { return "monocuda-pt-b200 0.1.0 (sm_100a)"; }

const char* mc_status_string(mc_status s) {
    switch (s) {
        case MC_OK: return "ok";
        case MC_ERR_INVALID: return "invalid argument";
        case MC_ERR_CUDA: return "CUDA error";
        case MC_ERR_OOM: return "out of device memory";
        case MC_ERR_STACK_OVERFLOW: return "traversal stack overflow";
        case MC_ERR_QUEUE_OVERFLOW: return "queue overflow";
        case MC_ERR_TIMEOUT: return "device wait timed out";
        case MC_ERR_BUDGET: return "request exceeds the memory budget";
        case MC_ERR_CANCELLED: return "cancelled";
        case MC_ERR_NOT_FOUND: return "not found";
        case MC_ERR_UNSUPPORTED: return "unsupported";
    }
    return "unknown status";
}

const char* mc_last_error(void) { return g_last_error; }

mc_status mc_context_create(int device, mc_context** out) {
    if (!out) return mc::set_error(MC_ERR_INVALID, "mc_context_create: null output");
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        cudaGetLastError();
        return mc::set_error(MC_ERR_UNSUPPORTED, "mc_context_create: no CUDA device (%s)", cudaGetErrorString(e));
    }
    if (device < 0 || device >= count) return mc::set_error(MC_ERR_INVALID, "mc_context_create: device %d out of range", device);
    if ((e = cudaSetDevice(device)) != cudaSuccess) return mc::cuda_error((int)e, "cudaSetDevice", __FILE__, __LINE__);
    cudaDeviceProp prop;
    if ((e = cudaGetDeviceProperties(&prop, device)) != cudaSuccess) return mc::cuda_error((int)e, "cudaGetDeviceProperties", __FILE__, __LINE__);
    if (prop.major < 10) return mc::set_error(MC_ERR_UNSUPPORTED, "mc_context_create: device %d is sm_%d%d; the library is compiled for sm_100a", device, prop.major, prop.minor);
    mc_context* ctx = new mc_context();
    ctx->device = device;
    ctx->sm_count = prop.multiProcessorCount;
    size_t counterBytes = (size_t)(MC_MAX_DEPTH_STATS + 1) * MC_COUNTERS_PER_DEPTH * sizeof(int);
    if (cudaMalloc(&ctx->d_error, sizeof(int)) != cudaSuccess || cudaMalloc(&ctx->d_wait_error, sizeof(int)) != cudaSuccess ||
        cudaMalloc(&ctx->d_counters, counterBytes) != cudaSuccess ||
        cudaMalloc(&ctx->d_stats, (2 * MC_MAX_DEPTH_STATS + 8) * sizeof(long long)) != cudaSuccess) {
        cudaGetLastError();
        mc_context_destroy(ctx);
        return mc::set_error(MC_ERR_OOM, "mc_context_create: device allocation failed");
    }
    cudaMemset(ctx->d_error, 0, sizeof(int));
    cudaMemset(ctx->d_wait_error, 0, sizeof(int));
    cudaMemset(ctx->d_counters, 0, counterBytes);
    *out = ctx;
    return MC_OK;
}

mc_status mc_context_destroy(mc_context* ctx) {
    if (!ctx) return MC_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream); else cudaDeviceSynchronize();
    cudaFree(ctx->d_error);
    cudaFree(ctx->d_wait_error);
    cudaFree(ctx->d_counters);
    cudaFree(ctx->d_stats);
    for (auto& b : ctx->scratch) mc::devbuf_free(b);
    mc::devbuf_free(ctx->wave.block);
    mc::devbuf_free(ctx->volume);
    cudaFree(ctx->rng_states);
    if (ctx->graph_exec) cudaGraphExecDestroy((cudaGraphExec_t)ctx->graph_exec);
    if (ctx->own_stream) {
        cudaStreamSynchronize(ctx->own_stream);
        cudaStreamDestroy(ctx->own_stream);
    }
    for (void* e : ctx->table_events)
        if (e) cudaEventDestroy((cudaEvent_t)e);
    cudaFree(ctx->d_table);
    if (ctx->h_tables) cudaFreeHost(ctx->h_tables);
    cudaFree(ctx->scene_of);
    if (ctx->staging) cudaFreeHost(ctx->staging);
    // the pool keeps the trees still alive; what it holds unused goes back
    mc::pool_trim(ctx->device);
    delete ctx;
    return MC_OK;
}

mc_status mc_context_set_stream(mc_context* ctx, void* stream) {
    if (!ctx) return mc::set_error(MC_ERR_INVALID, "mc_context_set_stream: null context");
    ctx->stream = (cudaStream_t)stream;
    return MC_OK;
}

mc_status mc_context_synchronize(mc_context* ctx) {
    if (!ctx) return mc::set_error(MC_ERR_INVALID, "mc_context_synchronize: null context");
    int flags = 0;
    cudaError_t e = cudaMemcpyAsync(&flags, ctx->d_wait_error, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return mc::cuda_error((int)e, "mc_context_synchronize", __FILE__, __LINE__);
    if (flags) {
        if ((e = cudaMemsetAsync(ctx->d_wait_error, 0, sizeof(int), ctx->stream)) != cudaSuccess)
            return mc::cuda_error((int)e, "mc_context_synchronize", __FILE__, __LINE__);
        return mc::set_error(MC_ERR_TIMEOUT, "mc_stream_wait_value: the flag was not set within the wait timeout");
    }
    return MC_OK;
}

mc_status mc_context_set_wait_timeout(mc_context* ctx, int64_t microseconds) {
    if (!ctx || microseconds < 0) return mc::set_error(MC_ERR_INVALID, "mc_context_set_wait_timeout: bad argument");
    ctx->wait_timeout_ns = microseconds == 0 ? 2000000000ll : (long long)microseconds * 1000ll;
    return MC_OK;
}

mc_status mc_stream_wait_value(mc_context* ctx, const uint32_t* d_flag, uint32_t value) {
    if (!ctx || !d_flag) return mc::set_error(MC_ERR_INVALID, "mc_stream_wait_value: null argument");
    mc::k_wait_value<<<1, 32, 0, ctx->stream>>>(d_flag, value, ctx->wait_timeout_ns, ctx->d_wait_error);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return mc::cuda_error((int)e, "mc_stream_wait_value", __FILE__, __LINE__);
    return MC_OK;
}

// PT:370-411: sampling tables (host) and a float4 texture, linear filtering,
// wrap in u, clamp in v, element-type reads, normalized coordinates.
// createImageTextureObject (PT:296-316): RGBA8 array, sRGB, bilinear,
// wrapped, normalised coordinates.
mc_status mc_image_texture_create(const uint8_t* rgba, int32_t width, int32_t height, uint64_t* texture) {
    if (!rgba || !texture || width <= 0 || height <= 0) return mc::set_error(MC_ERR_INVALID, "mc_image_texture_create: bad arguments");
    cudaChannelFormatDesc fmt = cudaCreateChannelDesc<uchar4>();
    cudaArray_t arr = nullptr;
    cudaError_t e = cudaMallocArray(&arr, &fmt, (size_t)width, (size_t)height);
    if (e == cudaSuccess)
        e = cudaMemcpy2DToArray(arr, 0, 0, rgba, (size_t)width * 4, (size_t)width * 4, (size_t)height, cudaMemcpyHostToDevice);
    cudaTextureObject_t tex = 0;
    if (e == cudaSuccess) {
        cudaResourceDesc res;
        std::memset(&res, 0, sizeof(res));
        res.resType = cudaResourceTypeArray;
        res.res.array.array = arr;
        cudaTextureDesc td;
        std::memset(&td, 0, sizeof(td));
        td.addressMode[0] = cudaAddressModeWrap;
        td.addressMode[1] = cudaAddressModeWrap;
        td.filterMode = cudaFilterModeLinear;
        td.readMode = cudaReadModeNormalizedFloat;
        td.normalizedCoords = 1;
        td.sRGB = 1;
        e = cudaCreateTextureObject(&tex, &res, &td, nullptr);
    }
    if (e != cudaSuccess) {
        if (arr) cudaFreeArray(arr);
        return mc::cuda_error((int)e, "mc_image_texture_create", __FILE__, __LINE__);
    }
    *texture = (uint64_t)tex;
    return MC_OK;
}

mc_status mc_image_texture_destroy(uint64_t texture) {
    if (!texture) return MC_OK;
    cudaResourceDesc res;
    cudaError_t e = cudaGetTextureObjectResourceDesc(&res, (cudaTextureObject_t)texture);
    if (e != cudaSuccess) return mc::cuda_error((int)e, "mc_image_texture_destroy", __FILE__, __LINE__);
    cudaDestroyTextureObject((cudaTextureObject_t)texture);
    if (res.resType == cudaResourceTypeArray && res.res.array.array) cudaFreeArray(res.res.array.array);
    return MC_OK;
}

}  // extern "C"

namespace mc {

// Walker's alias method with Vose's linear-time construction (M. D. Vose, "A
// linear algorithm for generating random numbers with a given distribution",
// IEEE TSE 17(9), 1991) over the texel weights of the column CDFs: entry i =
// (threshold, alias) with P(texel i) = (threshold_i + sum over j aliasing to i
// of (1 - threshold_j)) / n = w_i / sum w. Built in double precision.
void build_env_alias(const std::vector<float>& colCdf, int W, int H, std::vector<EnvAliasEntry>& table) {
    const size_t n = (size_t)W * H;
    table.assign(n, EnvAliasEntry{1.0f, 0});
    std::vector<double> p(n);
    double sum = 0.0;
    for (int row = 0; row < H; row++) {
        const float* cdf = &colCdf[(size_t)row * (W + 1)];
        for (int col = 0; col < W; col++) {
            const double w = (double)(cdf[col + 1] - cdf[col]);
            p[(size_t)row * W + col] = w > 0.0 ? w : 0.0;
            sum += p[(size_t)row * W + col];
        }
    }
    for (size_t i = 0; i < n; i++) table[i].alias = (int32_t)i;
    if (!(sum > 0.0)) return;
    std::vector<uint32_t> small, large;
    small.reserve(n);
    large.reserve(n);
    for (size_t i = 0; i < n; i++) {
        p[i] = p[i] * (double)n / sum;
        (p[i] < 1.0 ? small : large).push_back((uint32_t)i);
    }
    while (!small.empty() && !large.empty()) {
        const uint32_t s = small.back(), l = large.back();
        small.pop_back();
        table[s].threshold = (float)p[s];
        table[s].alias = (int32_t)l;
        p[l] = (p[l] + p[s]) - 1.0;
        if (p[l] < 1.0) {
            large.pop_back();
            small.push_back(l);
        }
    }
    // leftovers (rounding) keep their own texel with certainty
    for (uint32_t i : large) table[i] = EnvAliasEntry{1.0f, (int32_t)i};
    for (uint32_t i : small) table[i] = EnvAliasEntry{1.0f, (int32_t)i};
}

const void* env_alias_table(const mc_env_map& env) {
    if (!env.enabled || !env.col_cdf) return nullptr;
    std::lock_guard<std::mutex> lock(g_alias_mutex);
    auto it = g_alias_tables.find(env.col_cdf);
    return it == g_alias_tables.end() ? nullptr : it->second;
}

}  // namespace mc

extern "C" {

mc_status mc_env_create(const float* rgba, int32_t W, int32_t H, float intensity, float rotation, mc_env_map* out) {
    if (!out) return mc::set_error(MC_ERR_INVALID, "mc_env_create: null output");
    std::memset(out, 0, sizeof(*out));
    out->intensity = intensity;
    out->rotation = rotation;
    if (!rgba || W <= 0 || H <= 0) return MC_OK;  // disabled environment
    std::vector<float> rowCdf, colCdf;
    float total = 0.f;
    mc::build_env_tables(rgba, W, H, rowCdf, colCdf, total);
    cudaChannelFormatDesc desc = cudaCreateChannelDesc<float4>();
    cudaArray_t arr = nullptr;
    cudaError_t e;
    if ((e = cudaMallocArray(&arr, &desc, W, H)) != cudaSuccess) return mc::cuda_error((int)e, "cudaMallocArray", __FILE__, __LINE__);
    if ((e = cudaMemcpy2DToArray(arr, 0, 0, rgba, (size_t)W * sizeof(float4), (size_t)W * sizeof(float4), H, cudaMemcpyHostToDevice)) != cudaSuccess) {
        cudaFreeArray(arr);
        return mc::cuda_error((int)e, "cudaMemcpy2DToArray", __FILE__, __LINE__);
    }
    cudaResourceDesc res = {};
    res.resType = cudaResourceTypeArray;
    res.res.array.array = arr;
    cudaTextureDesc td = {};
    td.addressMode[0] = cudaAddressModeWrap;
    td.addressMode[1] = cudaAddressModeClamp;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 1;
    cudaTextureObject_t tex = 0;
    if ((e = cudaCreateTextureObject(&tex, &res, &td, nullptr)) != cudaSuccess) {
        cudaFreeArray(arr);
        return mc::cuda_error((int)e, "cudaCreateTextureObject", __FILE__, __LINE__);
    }
    std::vector<mc::EnvAliasEntry> alias;
    mc::build_env_alias(colCdf, W, H, alias);
    // one allocation: the column CDFs, then (16-byte aligned) the alias table
    const size_t colBytes = colCdf.size() * sizeof(float);
    const size_t aliasOffset = (colBytes + 15) & ~(size_t)15;
    float* dRow = nullptr; float* dCol = nullptr;
    if (cudaMalloc(&dRow, rowCdf.size() * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&dCol, aliasOffset + alias.size() * sizeof(mc::EnvAliasEntry)) != cudaSuccess) {
        cudaGetLastError();
        cudaDestroyTextureObject(tex);
        cudaFreeArray(arr);
        cudaFree(dRow);
        return mc::set_error(MC_ERR_OOM, "mc_env_create: device allocation failed");
    }
    char* dAlias = reinterpret_cast<char*>(dCol) + aliasOffset;
    if ((e = cudaMemcpy(dRow, rowCdf.data(), rowCdf.size() * sizeof(float), cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(dCol, colCdf.data(), colBytes, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(dAlias, alias.data(), alias.size() * sizeof(mc::EnvAliasEntry), cudaMemcpyHostToDevice)) !=
            cudaSuccess) {
        cudaDestroyTextureObject(tex);
        cudaFreeArray(arr);
        cudaFree(dRow);
        cudaFree(dCol);
        return mc::cuda_error((int)e, "mc_env_create: table upload", __FILE__, __LINE__);
    }
    {
        std::lock_guard<std::mutex> lock(g_alias_mutex);
        g_alias_tables[dCol] = dAlias;
    }
    out->texture = (uint64_t)tex;
    out->enabled = 1;
    out->row_cdf = dRow;
    out->col_cdf = dCol;
    out->width = W;
    out->height = H;
    out->total_weight = total;
    return MC_OK;
}

mc_status mc_env_destroy(mc_env_map* env) {
    if (!env || !env->enabled) return MC_OK;
    cudaResourceDesc res;
    if (cudaGetTextureObjectResourceDesc(&res, (cudaTextureObject_t)env->texture) == cudaSuccess) {
        cudaDestroyTextureObject((cudaTextureObject_t)env->texture);
        if (res.resType == cudaResourceTypeArray) cudaFreeArray(res.res.array.array);
    }
    cudaFree((void*)env->row_cdf);
    {
        std::lock_guard<std::mutex> lock(g_alias_mutex);
        g_alias_tables.erase(env->col_cdf);
    }
    cudaFree((void*)env->col_cdf);
    std::memset(env, 0, sizeof(*env));
    return MC_OK;
}

}  // extern "C"
