// mc_ingest.cu - scene ingestion on the device: the per-triangle part of
// finalizeScene (PT:1930-1987: bounding boxes, the emissive-triangle light
// list in triangle order) and main()'s hot/cold split (PT:4276-4289), as
// kernels over a device array of AoS triangles.
//
// Compiled with IEEE arithmetic and no contraction (-fmad=false, IEEE division
// and square root): the light areas and normals must equal the reference's
// host computation bit for bit.
//
// The work is a byte shuffle bound by HBM: 224 B read and 228 B written per
// triangle. A block stages a tile of 128 triangles in shared memory with
// coalesced 16-byte loads, computes the boxes there, and writes the hot and
// cold tiles with coalesced 16-byte stores. The light list needs triangle
// order, so each tile only counts its emissive triangles; a one-block scan
// turns the counts into offsets and a third kernel, which returns at once for
// tiles without lights, writes the lights.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cstdint>

#include "mc_internal.h"

namespace mc {
namespace {

constexpr int kTile = 128;                  // triangles per block
constexpr int kThreads = 256;
constexpr int kTriWords = (int)sizeof(mc_triangle) / 4;       // 56
constexpr int kHotWords = (int)sizeof(mc_triangle_hot) / 4;   // 9
constexpr int kColdWords = (int)sizeof(mc_triangle_cold) / 4; // 48
constexpr int kScanThreads = 1024;

static_assert(sizeof(mc_triangle) == 224 && sizeof(mc_triangle_cold) == 192 && sizeof(mc_triangle_hot) == 36,
              "ingest word maps assume the reference layouts");
static_assert(offsetof(mc_triangle, uv0) == 36 && offsetof(mc_triangle, mat) == 96 && offsetof(mc_triangle, aabb) == 192,
              "triangle layout");
static_assert(offsetof(mc_triangle_cold, mat) == 64 && offsetof(mc_triangle_cold, aabb) == 160, "cold layout");

// Word k (0..47) of a cold record, from the staged triangle words and its box:
// [0,15) uv0..n2 = triangle words 9..23; 15 the padding before the material
// (zero, as a value-initialised record); [16,40) the material = triangle words
// 24..47; [40,48) the box.
__device__ __forceinline__ uint32_t cold_word(const uint32_t* tri, const uint32_t* box, int k) {
    if (k < 15) return tri[9 + k];
    if (k == 15) return 0u;
    if (k < 40) return tri[24 + (k - 16)];
    return box[k - 40];
}

__global__ void __launch_bounds__(kThreads) k_ingest_split(const mc_triangle* __restrict__ tris, int n,
                                                           mc_triangle_hot* __restrict__ hot,
                                                           mc_triangle_cold* __restrict__ cold,
                                                           int* __restrict__ tileCount, int* __restrict__ flags) {
    __shared__ __align__(16) uint32_t sTri[kTile * kTriWords];
    __shared__ __align__(16) uint32_t sBox[kTile * 8];
    const long long base = (long long)blockIdx.x * kTile;
    const int cnt = (int)min((long long)kTile, (long long)n - base);

    // Stage the tile: cnt * 224 bytes, always a whole number of 16-byte words.
    {
        const int4* src = reinterpret_cast<const int4*>(tris + base);
        int4* dst = reinterpret_cast<int4*>(sTri);
        const int v4 = cnt * (kTriWords / 4);
        for (int j = threadIdx.x; j < v4; j += kThreads) dst[j] = __ldcs(src + j);
    }
    __syncthreads();

    // PT:651-655 calculate_bounding_box: min/max of the vertices -/+ 1e-3.
    bool emissive = false, medium = false, grid = false;
    if (threadIdx.x < cnt) {
        const mc_triangle& t = *reinterpret_cast<const mc_triangle*>(sTri + threadIdx.x * kTriWords);
        const float eps = 1e-3f;
        float* b = reinterpret_cast<float*>(sBox + threadIdx.x * 8);
        b[0] = fminf(t.v0.x, fminf(t.v1.x, t.v2.x)) - eps;
        b[1] = fminf(t.v0.y, fminf(t.v1.y, t.v2.y)) - eps;
        b[2] = fminf(t.v0.z, fminf(t.v1.z, t.v2.z)) - eps;
        b[3] = 0.f;
        b[4] = fmaxf(t.v0.x, fmaxf(t.v1.x, t.v2.x)) + eps;
        b[5] = fmaxf(t.v0.y, fmaxf(t.v1.y, t.v2.y)) + eps;
        b[6] = fmaxf(t.v0.z, fmaxf(t.v1.z, t.v2.z)) + eps;
        b[7] = 0.f;
        emissive = t.mat.type == MC_MAT_EMISSIVE;
        medium = t.mat.type == MC_MAT_ISOTROPIC;
        grid = medium && t.mat.density_grid != nullptr;
    }
    const int lights = __syncthreads_count(emissive);
    const int anyMedium = __syncthreads_or(medium);
    const int anyGrid = __syncthreads_or(grid);
    if (threadIdx.x == 0) {
        tileCount[blockIdx.x] = lights;
        if (anyMedium) atomicOr(flags, anyGrid ? MC_MEDIUM_ANY | MC_MEDIUM_GRID : MC_MEDIUM_ANY);
    }

    // Hot records: the first 9 words of each triangle.
    if (cnt == kTile) {
        int4* dst = reinterpret_cast<int4*>(hot + base);
        for (int j = threadIdx.x; j < kTile * kHotWords / 4; j += kThreads) {
            uint32_t w[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int k = 4 * j + q;
                w[q] = sTri[(k / kHotWords) * kTriWords + k % kHotWords];
            }
            __stcs(dst + j, make_int4((int)w[0], (int)w[1], (int)w[2], (int)w[3]));
        }
    } else {
        uint32_t* dst = reinterpret_cast<uint32_t*>(hot + base);
        for (int k = threadIdx.x; k < cnt * kHotWords; k += kThreads)
            dst[k] = sTri[(k / kHotWords) * kTriWords + k % kHotWords];
    }
    // Cold records: 12 16-byte words each, none straddling two triangles.
    {
        int4* dst = reinterpret_cast<int4*>(cold + base);
        for (int j = threadIdx.x; j < cnt * (kColdWords / 4); j += kThreads) {
            const int tri = j / (kColdWords / 4);
            const int k0 = 4 * (j % (kColdWords / 4));
            const uint32_t* tw = sTri + tri * kTriWords;
            const uint32_t* bw = sBox + tri * 8;
            __stcs(dst + j, make_int4((int)cold_word(tw, bw, k0), (int)cold_word(tw, bw, k0 + 1),
                                      (int)cold_word(tw, bw, k0 + 2), (int)cold_word(tw, bw, k0 + 3)));
        }
    }
}

// Exclusive scan of the per-tile light counts (one block; the counts are few
// compared with the triangles). total[0] receives the light count.
__global__ void __launch_bounds__(kScanThreads) k_ingest_scan(const int* __restrict__ tileCount, int tiles,
                                                               int* __restrict__ tileOffset, int* __restrict__ total) {
    __shared__ int warpSum[kScanThreads / 32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int start = 0; start < tiles; start += kScanThreads) {
        const int i = start + threadIdx.x;
        const int v = i < tiles ? tileCount[i] : 0;
        int x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warpSum[warp] = x;
        __syncthreads();
        if (warp == 0) {
            int s = warpSum[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, s, o);
                if (lane >= o) s += y;
            }
            warpSum[lane] = s;  // inclusive over warps
        }
        __syncthreads();
        const int before = carry + (warp > 0 ? warpSum[warp - 1] : 0) + x - v;
        if (i < tiles) tileOffset[i] = before;
        __syncthreads();
        if (threadIdx.x == kScanThreads - 1) carry = before + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) total[0] = carry;
}

// PT:1972-1985: one Light per emissive triangle, in triangle order. The area
// vector, its length and the normal follow the host vec3 arithmetic:
// (y*o.z - z*o.y, ...), sqrt(x*x + y*y + z*z), then each component / length.
__global__ void __launch_bounds__(kTile) k_ingest_lights(const mc_triangle* __restrict__ tris, int n,
                                                         const int* __restrict__ tileCount,
                                                         const int* __restrict__ tileOffset,
                                                         mc_light* __restrict__ lights) {
    if (tileCount[blockIdx.x] == 0) return;
    __shared__ int warpCount[kTile / 32];
    const long long i = (long long)blockIdx.x * kTile + threadIdx.x;
    const bool em = i < n && tris[i].mat.type == MC_MAT_EMISSIVE;
    const unsigned m = __ballot_sync(0xffffffffu, em);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) warpCount[warp] = __popc(m);
    __syncthreads();
    if (!em) return;
    int rank = __popc(m & ((1u << lane) - 1u));
    for (int w = 0; w < warp; w++) rank += warpCount[w];
    const mc_triangle& t = tris[i];
    const float e1x = t.v1.x - t.v0.x, e1y = t.v1.y - t.v0.y, e1z = t.v1.z - t.v0.z;
    const float e2x = t.v2.x - t.v0.x, e2y = t.v2.y - t.v0.y, e2z = t.v2.z - t.v0.z;
    const float ax = e1y * e2z - e1z * e2y;
    const float ay = e1z * e2x - e1x * e2z;
    const float az = e1x * e2y - e1y * e2x;
    const float len = sqrtf(ax * ax + ay * ay + az * az);
    mc_light L;
    L.tri.v0 = t.v0; L.tri.v1 = t.v1; L.tri.v2 = t.v2;
    L.emitted = t.mat.emitted;
    L.area = 0.5f * len;
    L.normal = mc_vec3{ax / len, ay / len, az / len};
    lights[tileOffset[blockIdx.x] + rank] = L;
}

__global__ void k_ingest_spheres(const mc_sphere* __restrict__ sph, int ns, int* __restrict__ flags) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ns; i += gridDim.x * blockDim.x)
        if (sph[i].mat.type == MC_MAT_ISOTROPIC)
            atomicOr(flags, sph[i].mat.density_grid ? MC_MEDIUM_ANY | MC_MEDIUM_GRID : MC_MEDIUM_ANY);
}

bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

}  // namespace
}  // namespace mc

#define MC_CUDA(call)                                                                      \
    do {                                                                                   \
        cudaError_t e__ = (call);                                                          \
        if (e__ != cudaSuccess) return mc::cuda_error((int)e__, #call, __FILE__, __LINE__); \
    } while (0)

extern "C" mc_status mc_scene_ingest(mc_context* ctx, const mc_triangle* tris, int32_t n, const mc_sphere* spheres,
                                     int32_t n_sph, mc_triangle_hot* hot, mc_triangle_cold* cold, mc_light* lights,
                                     int32_t* light_count, int32_t* has_medium) {
    using namespace mc;
    if (!ctx || n < 0 || n_sph < 0 || (n > 0 && (!tris || !hot || !cold)) || (n_sph > 0 && !spheres))
        return set_error(MC_ERR_INVALID, "mc_scene_ingest: bad arguments");
    if (n > 0 && (!aligned16(tris) || !aligned16(hot) || !aligned16(cold)))
        return set_error(MC_ERR_INVALID, "mc_scene_ingest: tris, hot and cold must be 16-byte aligned device arrays");
    const int tiles = (int)(((long long)n + kTile - 1) / kTile);
    // scratch: flags, light total, then tile counts and offsets
    mc_status st = devbuf_reserve(ctx->scratch[0], (size_t)(4 + 2 * (long long)tiles) * sizeof(int));
    if (st != MC_OK) return st;
    int* flags = (int*)ctx->scratch[0].ptr;
    int* total = flags + 1;
    int* tileCount = flags + 4;
    int* tileOffset = tileCount + tiles;
    MC_CUDA(cudaMemsetAsync(flags, 0, 4 * sizeof(int), ctx->stream));
    if (n > 0) {
        k_ingest_split<<<tiles, kThreads, 0, ctx->stream>>>(tris, n, hot, cold, tileCount, flags);
        MC_CUDA(cudaGetLastError());
        k_ingest_scan<<<1, kScanThreads, 0, ctx->stream>>>(tileCount, tiles, tileOffset, total);
        MC_CUDA(cudaGetLastError());
        if (lights) {
            k_ingest_lights<<<tiles, kTile, 0, ctx->stream>>>(tris, n, tileCount, tileOffset, lights);
            MC_CUDA(cudaGetLastError());
        }
    }
    if (n_sph > 0) {
        k_ingest_spheres<<<std::min((n_sph + 255) / 256, 4 * ctx->sm_count), 256, 0, ctx->stream>>>(spheres, n_sph, flags);
        MC_CUDA(cudaGetLastError());
    }
    int h[2] = {0, 0};
    MC_CUDA(cudaMemcpyAsync(h, flags, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    MC_CUDA(cudaStreamSynchronize(ctx->stream));
    if (light_count) *light_count = h[1];
    if (has_medium) *has_medium = h[0] & (MC_MEDIUM_ANY | MC_MEDIUM_GRID);
    return MC_OK;
}

extern "C" mc_status mc_scene_ingest_host(mc_context* ctx, const mc_triangle* tris, int32_t n, const mc_sphere* spheres,
                                          int32_t n_sph, mc_triangle_hot* hot, mc_triangle_cold* cold, mc_light* lights,
                                          int32_t* light_count, int32_t* has_medium) {
    using namespace mc;
    if (!ctx || n < 0 || (n > 0 && !tris)) return set_error(MC_ERR_INVALID, "mc_scene_ingest_host: bad arguments");
    mc_triangle* dTri = nullptr;
    if (n > 0 && cudaMalloc(&dTri, (size_t)n * sizeof(mc_triangle)) != cudaSuccess) {
        cudaGetLastError();
        return set_error(MC_ERR_OOM, "mc_scene_ingest_host: device allocation failed");
    }
    mc_status st = upload_host(ctx, dTri, tris, (size_t)n * sizeof(mc_triangle));
    if (st == MC_OK) st = mc_scene_ingest(ctx, dTri, n, spheres, n_sph, hot, cold, lights, light_count, has_medium);
    cudaFree(dTri);
    return st;
}
