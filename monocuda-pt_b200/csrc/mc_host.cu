// mc_host.cu - host-memory entry point and the launch-parameter autotuner.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cstring>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "mc_internal.h"

#define MC_CUDA(call)                                                                      \
    do {                                                                                   \
        cudaError_t e__ = (call);                                                          \
        if (e__ != cudaSuccess) return mc::cuda_error((int)e__, #call, __FILE__, __LINE__); \
    } while (0)

namespace mc {
mc_status ensure_wave(mc_context* ctx, int capacity);

namespace {
constexpr size_t kStagePiece = (size_t)4 << 20;    // bytes per staging buffer
constexpr size_t kStageDirect = (size_t)32 << 20;  // smaller copies go straight from pageable memory
}  // namespace

// A pageable cudaMemcpy moves about 11 GB/s through the driver's own staging;
// T host threads, each filling two pinned pieces of its own in turn while the
// DMA of the other runs on its own stream, reach about 40 GB/s (8 threads,
// 4 MB pieces) against 55 GB/s from pinned memory. The pinned buffers stay
// with the context: allocating them costs about 0.5 ms per MB.
mc_status upload_host(mc_context* ctx, void* dst, const void* src, size_t bytes) {
    if (bytes == 0) return MC_OK;
    cudaPointerAttributes attr;
    bool pinned = false;
    if (cudaPointerGetAttributes(&attr, src) == cudaSuccess) pinned = attr.type == cudaMemoryTypeHost;
    else cudaGetLastError();
    if (bytes < kStageDirect || pinned) {
        cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        return e == cudaSuccess ? MC_OK : cuda_error((int)e, "upload", __FILE__, __LINE__);
    }
    const unsigned hw = std::thread::hardware_concurrency();
    const int T = (int)std::max(1u, std::min(8u, hw ? hw : 1u));
    const size_t need = 2 * (size_t)T * kStagePiece;
    if (ctx->staging_bytes < need) {
        if (ctx->staging) cudaFreeHost(ctx->staging);
        ctx->staging = nullptr;
        ctx->staging_bytes = 0;
        if (cudaHostAlloc(&ctx->staging, need, cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            ctx->staging = nullptr;
            return set_error(MC_ERR_OOM, "upload: pinned staging allocation failed");
        }
        ctx->staging_bytes = need;
    }
    // work queued earlier on the context's stream may still read dst
    cudaError_t e0 = cudaStreamSynchronize(ctx->stream);
    if (e0 != cudaSuccess) return cuda_error((int)e0, "upload", __FILE__, __LINE__);
    std::vector<cudaError_t> err((size_t)T, cudaSuccess);
    std::vector<std::thread> th;
    const size_t share = (bytes + T - 1) / T;
    for (int k = 0; k < T; k++) {
        th.emplace_back([&, k]() {
            cudaError_t e = cudaSetDevice(ctx->device);
            cudaStream_t s = nullptr;
            cudaEvent_t ev[2] = {nullptr, nullptr};
            if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming);
            const size_t lo = std::min(bytes, share * k), hi = std::min(bytes, share * (k + 1));
            char* buf[2] = {(char*)ctx->staging + (2 * k) * kStagePiece, (char*)ctx->staging + (2 * k + 1) * kStagePiece};
            bool used[2] = {false, false};
            int slot = 0;
            for (size_t o = lo; o < hi && e == cudaSuccess; o += kStagePiece) {
                const size_t len = std::min(kStagePiece, hi - o);
                if (used[slot]) e = cudaEventSynchronize(ev[slot]);
                if (e != cudaSuccess) break;
                std::memcpy(buf[slot], (const char*)src + o, len);
                e = cudaMemcpyAsync((char*)dst + o, buf[slot], len, cudaMemcpyHostToDevice, s);
                if (e == cudaSuccess) e = cudaEventRecord(ev[slot], s);
                used[slot] = true;
                slot ^= 1;
            }
            if (s) {
                cudaError_t e2 = cudaStreamSynchronize(s);
                if (e == cudaSuccess) e = e2;
                cudaStreamDestroy(s);
            }
            for (cudaEvent_t x : ev)
                if (x) cudaEventDestroy(x);
            err[(size_t)k] = e;
        });
    }
    for (auto& t : th) t.join();
    for (cudaError_t e : err)
        if (e != cudaSuccess) return cuda_error((int)e, "upload", __FILE__, __LINE__);
    return MC_OK;
}
}  // namespace mc

extern "C" {

// The whole reference flow from host arrays (PT:4223-4336): upload of the AoS
// triangles, then on the device finalize + light list + hot/cold split
// (mc_scene_ingest_host), BVH build, render, accumulation read-back.
mc_status mc_render_host(mc_context* ctx, const mc_triangle* tris, int32_t n_tri, const mc_sphere* spheres, int32_t n_sph,
                         const mc_env_map* env, const mc_render_params* params, float* accum_host, mc_render_stats* stats) {
    if (!ctx || !params || !accum_host || n_tri < 0 || n_sph < 0 || (n_tri > 0 && !tris) || (n_sph > 0 && !spheres))
        return mc::set_error(MC_ERR_INVALID, "mc_render_host: bad argument");
    if (n_tri + n_sph == 0) return mc::set_error(MC_ERR_INVALID, "mc_render_host: the scene has no primitives");
    const size_t nt = (size_t)(n_tri > 0 ? n_tri : 1);
    mc_triangle_hot* dHot = nullptr; mc_triangle_cold* dCold = nullptr; mc_sphere* dSph = nullptr; mc_light* dL = nullptr;
    float* dAcc = nullptr;
    size_t accBytes = (size_t)params->width * params->height * 3 * sizeof(float);
    auto cleanup = [&]() { cudaFree(dHot); cudaFree(dCold); cudaFree(dSph); cudaFree(dL); cudaFree(dAcc); };
    if (cudaMalloc(&dHot, nt * sizeof(mc_triangle_hot)) != cudaSuccess ||
        cudaMalloc(&dCold, nt * sizeof(mc_triangle_cold)) != cudaSuccess ||
        cudaMalloc(&dSph, (size_t)(n_sph > 0 ? n_sph : 1) * sizeof(mc_sphere)) != cudaSuccess ||
        cudaMalloc(&dL, nt * sizeof(mc_light)) != cudaSuccess || cudaMalloc(&dAcc, accBytes) != cudaSuccess) {
        cudaGetLastError();
        cleanup();
        return mc::set_error(MC_ERR_OOM, "mc_render_host: device allocation failed");
    }
    if (n_sph) cudaMemcpyAsync(dSph, spheres, (size_t)n_sph * sizeof(mc_sphere), cudaMemcpyHostToDevice, ctx->stream);
    cudaMemcpyAsync(dAcc, accum_host, accBytes, cudaMemcpyHostToDevice, ctx->stream);
    int32_t nl = 0, hasMedium = 0;
    mc_status st0 = mc_scene_ingest_host(ctx, tris, n_tri, dSph, n_sph, dHot, dCold, dL, &nl, &hasMedium);
    if (st0 != MC_OK) {
        cleanup();
        return st0;
    }
    mc_scene_view view;
    std::memset(&view, 0, sizeof(view));
    view.spheres = dSph; view.sphere_count = n_sph;
    view.tri_hot = dHot; view.tri_cold = dCold; view.triangle_count = n_tri;
    view.lights = dL; view.light_count = nl;
    view.has_medium = hasMedium;
    if (env) view.env = *env;
    mc_bvh* bvh = nullptr;
    mc_bvh_build_opts opts;
    std::memset(&opts, 0, sizeof(opts));
    opts.layout = MC_BVH_LAYOUT_WIDE4;  // the faster layout; hits identical to the binary one
    mc_status st = mc_bvh_build(ctx, &view, &opts, &bvh);
    if (st == MC_OK) st = mc_render_wavefront(ctx, bvh, &view, params, dAcc, stats);
    if (st == MC_OK) {
        cudaError_t e = cudaMemcpyAsync(accum_host, dAcc, accBytes, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) st = mc::cuda_error((int)e, "mc_render_host read-back", __FILE__, __LINE__);
    }
    mc_bvh_free(bvh);
    cleanup();
    return st;
}

// Picks the launch configuration by timing real waves of this render (full
// resolution, the scene's own BVH), in stages: the trace variant and refill
// threshold; the trace block shape and stack; the samples per wave (the queue
// capacity); CUDA graph replay. In each stage every candidate runs once
// untimed, then up to three timed rounds in turn, each keeping its fastest
// time per sample. Results are cached per (device, layout, scene size class,
// image size class, spp class): later calls in the same class return at once.
// None of the choices changes the image. budget_ms bounds the tuning time
// (0 = 2000); stages not reached by then keep their defaults.
mc_status mc_autotune(mc_context* ctx, const mc_bvh* bvh, const mc_scene_view* scene, mc_render_params* params, int32_t budget_ms) {
    if (!ctx || !bvh || !scene || !params) return mc::set_error(MC_ERR_INVALID, "mc_autotune: null argument");
    if (params->width < 1 || params->height < 1) return mc::set_error(MC_ERR_INVALID, "mc_autotune: empty image");
    if (budget_ms <= 0) budget_ms = 2000;
    struct Choice { int persistent, refill, graph, spw, threads, stack; };
    static std::mutex mu;
    static std::map<std::array<long long, 5>, Choice> cache;
    auto log2c = [](long long v) { int b = 0; while (v > 1) { v >>= 1; b++; } return (long long)b; };
    const int k = mc::wave_samples(params);
    const long long pixels = (long long)params->width * params->height;
    const std::array<long long, 5> key = {(long long)ctx->device, (long long)bvh->layout, log2c(bvh->n), log2c(pixels),
                                          log2c(std::max(1, params->spp))};
    auto apply = [&](const Choice& c) {
        params->persistent = c.persistent;
        params->refill_threshold = c.refill;
        params->use_graph = c.graph;
        params->samples_per_wave = c.spw;
        params->trace_threads = c.threads;
        params->stack_entries = c.stack;
    };
    {
        std::lock_guard<std::mutex> lock(mu);
        auto it = cache.find(key);
        if (it != cache.end()) {
            apply(it->second);
            return MC_OK;
        }
    }
    mc_render_params probe = *params;
    probe.first_sample = 0;
    probe.instrument = 0;
    float* dAcc = nullptr;
    if (cudaMalloc(&dAcc, (size_t)pixels * 3 * sizeof(float)) != cudaSuccess) {
        cudaGetLastError();
        return mc::set_error(MC_ERR_OOM, "mc_autotune: allocation failed");
    }
    auto t0 = std::chrono::steady_clock::now();
    auto elapsed = [&]() { return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count(); };
    // one wave of c.spw samples; *ms: host time per sample
    auto run = [&](const Choice& c, float* ms) -> mc_status {
        probe.persistent = c.persistent;
        probe.refill_threshold = c.refill;
        probe.use_graph = c.graph;
        probe.spp = c.spw;
        probe.samples_per_wave = c.spw;
        probe.trace_threads = c.threads;
        probe.stack_entries = c.stack;
        mc_render_stats rs;
        auto a = std::chrono::steady_clock::now();
        mc_status st = mc_render_wavefront(ctx, bvh, scene, &probe, dAcc, &rs);
        if (cudaDeviceSynchronize() != cudaSuccess && st == MC_OK) st = mc::set_error(MC_ERR_CUDA, "mc_autotune: render failed");
        if (ms) *ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - a).count() / c.spw;
        return st;
    };
    // every candidate once (kernel loads, buffers, graph capture), then timed rounds; returns the fastest
    auto tune = [&](const std::vector<Choice>& cs, size_t* bestIdx) -> mc_status {
        std::vector<float> best(cs.size(), 1e30f);
        for (const Choice& c : cs) {
            mc_status st = run(c, nullptr);
            if (st != MC_OK) return st;
        }
        for (int round = 0; round < 3 && elapsed() < budget_ms; round++) {
            for (size_t i = 0; i < cs.size(); i++) {
                float ms = 0.f;
                mc_status st = run(cs[i], &ms);
                if (st != MC_OK) return st;
                best[i] = std::min(best[i], ms);
            }
        }
        size_t b = 0;
        for (size_t i = 1; i < cs.size(); i++)
            if (best[i] < best[b]) b = i;
        *bestIdx = best[b] < 1e30f ? b : 0;
        return MC_OK;
    };
    Choice bestC = {params->persistent, params->refill_threshold > 0 ? params->refill_threshold : 8, params->use_graph,
                    k, 256, 0};
    mc_status st = MC_OK;
    size_t b = 0;
    // 1: persistence and refill threshold
    std::vector<Choice> cands;
    for (int r : {8, 4, 12, 16, 24}) cands.push_back({1, r, 0, k, 256, 0});
    cands.push_back({0, 8, 0, k, 256, 0});
    if ((st = tune(cands, &b)) == MC_OK) bestC = cands[b];
    // 2: 128-thread blocks with the stack the 4-wide tree needs (3 entries per
    // level, rounded up to 8): 7 blocks per SM fit in shared memory up to 56
    // entries (persistent renders of wide layouts without density grids)
    const int need = bvh->wide_levels > 0 ? ((3 * bvh->wide_levels + 7) / 8) * 8 : 999;
    if (st == MC_OK && elapsed() < budget_ms && bestC.persistent && bvh->layout != MC_BVH_LAYOUT_BINARY && need <= 56 &&
        !(scene->has_medium & MC_MEDIUM_GRID) && params->intersector == MC_ISECT_REFERENCE) {
        Choice small = bestC;
        small.threads = 128;
        small.stack = need;
        std::vector<Choice> pair = {bestC, small};
        if ((st = tune(pair, &b)) == MC_OK) bestC = pair[b];
    }
    // 3: queue capacity (samples per wave): the automatic choice against twice it
    const long long maxPaths = 64ll << 20;
    if (st == MC_OK && elapsed() < budget_ms && params->rng == MC_RNG_PHILOX && params->samples_per_wave == 0 &&
        2 * k <= params->spp && pixels * 2 * k <= maxPaths) {
        Choice twice = bestC;
        twice.spw = 2 * k;
        std::vector<Choice> pair = {bestC, twice};
        if ((st = tune(pair, &b)) == MC_OK) bestC = pair[b];
    }
    // 4: graph replay of the winner against the winner as launched
    if (st == MC_OK && elapsed() < budget_ms) {
        Choice g = bestC;
        g.graph = 1;
        std::vector<Choice> pair = {bestC, g};
        if ((st = tune(pair, &b)) == MC_OK) bestC = pair[b];
    }
    cudaFree(dAcc);
    if (st != MC_OK) return st;
    // an explicit samples_per_wave of the caller stays as it was
    if (params->samples_per_wave != 0) bestC.spw = params->samples_per_wave;
    else if (bestC.spw == k) bestC.spw = 0;
    apply(bestC);
    std::lock_guard<std::mutex> lock(mu);
    cache[key] = bestC;
    return MC_OK;
}

}  // extern "C"
