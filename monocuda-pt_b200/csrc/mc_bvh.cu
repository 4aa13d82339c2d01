// mc_bvh.cu - LBVH build on the device, for one scene or a batch of scenes.
//
//   primitive bounds + centroids + scene bounds  (finalizeScene, PT:1930-1971)
//   30-bit Morton codes                          (morton3D, PT:913-935; host IEEE math in the reference)
//   stable onesweep LSD radix sort               (replaces the host std::sort, PT:4223-4226)
//   Karras radix tree                            (delta/determineRange/findSplit, PT:1337-1447)
//   bottom-up refit with per-node arrival counters (refitBoundsKernel, PT:1398-1415), which writes
//   the boxes straight into the traversal layout (children's boxes stored in the parent)
//   optional 4-wide collapse.
//
// A batch of scenes is built by the same launches: every kernel maps a global
// primitive / node index to its scene ("segment") and the segment-local index
// the reference's algorithm works on; each segment gets its own root. The sort
// orders by (segment, Morton code): a 30-bit pass sequence on the codes, then a
// stable pass on the segment id.
//
// This file is compiled WITHOUT fast math and with -fmad=false: the reference
// computes bounds and Morton codes on the host with IEEE single precision and
// no contraction, and the codes must match bit for bit.
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "mc_internal.h"

namespace {

constexpr int kBlock = 256;
constexpr int kRadixBits = 8;
constexpr int kRadix = 256;
constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 16;
constexpr int kTile = kSortThreads * kSortItems;
constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagInc = 2u << 30;
constexpr uint32_t kCountMask = (1u << 30) - 1;
constexpr long long kSpinLimit = 1ll << 22;

#define MC_CUDA(call)                                                                      \
    do {                                                                                   \
        cudaError_t e__ = (call);                                                          \
        if (e__ != cudaSuccess) return mc::cuda_error((int)e__, #call, __FILE__, __LINE__); \
    } while (0)

struct Box {
    float lx, ly, lz, hx, hy, hz;
};

// One scene of a build: its primitive arrays and where its primitives and
// internal nodes start in the batch-wide arrays.
struct Seg {
    const mc_sphere* sph;
    const mc_triangle_hot* hot;
    int ns, nt;
    int primOff;   // first global primitive (leaf) index
    int intOff;    // first global internal-node index (= primOff - segment index)
};

__device__ __forceinline__ int seg_of_prim(const Seg* seg, int nseg, int g) {
    int lo = 0, hi = nseg - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (seg[mid].primOff <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ int seg_of_internal(const Seg* seg, int nseg, int g) {
    int lo = 0, hi = nseg - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (seg[mid].intOff <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ Box merge_box(const Box& a, const Box& b) {  // PT:1456-1465 merge
    Box m;
    m.hx = fmaxf(a.hx, b.hx);
    m.hy = fmaxf(a.hy, b.hy);
    m.hz = fmaxf(a.hz, b.hz);
    m.lx = fminf(a.lx, b.lx);
    m.ly = fminf(a.ly, b.ly);
    m.lz = fminf(a.lz, b.lz);
    return m;
}

// Ordered-integer encoding so atomicMin/atomicMax on ints order floats.
__device__ __forceinline__ int float_to_ordered(float f) {
    int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7FFFFFFF;
}
__host__ __device__ __forceinline__ float ordered_to_float(int i) {
#ifdef __CUDA_ARCH__
    return __int_as_float(i >= 0 ? i : i ^ 0x7FFFFFFF);
#else
    int j = i >= 0 ? i : i ^ 0x7FFFFFFF;
    float f;
    memcpy(&f, &j, 4);
    return f;
#endif
}

// Bounds and centroid of every primitive (per scene: spheres first, then
// triangles, PT:1955-1971). Sphere: calculate_bounding_box / calculateCentroid
// (PT:850-869). Triangle: calculate_bounding_box with eps 1e-3 / (v0+v1+v2)/3
// (PT:647-656). Scene bounds per segment (min/max are exact in any order).
__global__ void k_prim_bounds(const Seg* __restrict__ seg, int nseg, int n, mc_aabb* __restrict__ bounds,
                              float4* __restrict__ centroids, int* __restrict__ scene) {
    int g = blockIdx.x * blockDim.x + threadIdx.x;
    Box b = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
    bool valid = g < n;
    int s = valid ? seg_of_prim(seg, nseg, g) : 0;
    if (valid) {
        const Seg& S = seg[s];
        int i = g - S.primOff;
        float cx, cy, cz;
        if (i < S.ns) {
            const mc_sphere& sp = S.sph[i];
            float r = sp.radius;
            Box b0 = {sp.center.x - r, sp.center.y - r, sp.center.z - r, sp.center.x + r, sp.center.y + r, sp.center.z + r};
            if (sp.is_moving) {
                Box b1 = {sp.center1.x - r, sp.center1.y - r, sp.center1.z - r, sp.center1.x + r, sp.center1.y + r, sp.center1.z + r};
                b = merge_box(b0, b1);
                cx = (sp.center.x + sp.center1.x) * 0.5f;
                cy = (sp.center.y + sp.center1.y) * 0.5f;
                cz = (sp.center.z + sp.center1.z) * 0.5f;
            } else {
                b = b0;
                cx = sp.center.x; cy = sp.center.y; cz = sp.center.z;
            }
        } else {
            const mc_triangle_hot& t = S.hot[i - S.ns];
            const float eps = 1e-3f;
            b.lx = fminf(t.v0.x, fminf(t.v1.x, t.v2.x)) - eps;
            b.ly = fminf(t.v0.y, fminf(t.v1.y, t.v2.y)) - eps;
            b.lz = fminf(t.v0.z, fminf(t.v1.z, t.v2.z)) - eps;
            b.hx = fmaxf(t.v0.x, fmaxf(t.v1.x, t.v2.x)) + eps;
            b.hy = fmaxf(t.v0.y, fmaxf(t.v1.y, t.v2.y)) + eps;
            b.hz = fmaxf(t.v0.z, fmaxf(t.v1.z, t.v2.z)) + eps;
            cx = (t.v0.x + t.v1.x + t.v2.x) / 3.0f;
            cy = (t.v0.y + t.v1.y + t.v2.y) / 3.0f;
            cz = (t.v0.z + t.v1.z + t.v2.z) / 3.0f;
        }
        mc_aabb a;
        a.lo = mc_vec3{b.lx, b.ly, b.lz};
        a.pad0 = 0.f;
        a.hi = mc_vec3{b.hx, b.hy, b.hz};
        a.pad1 = 0.f;
        bounds[g] = a;
        centroids[g] = make_float4(cx, cy, cz, __int_as_float(s));
    }
    int* sb = scene + 6 * s;
    int s0 = __shfl_sync(0xffffffffu, s, 0);
    if (__all_sync(0xffffffffu, s == s0)) {
        for (int off = 16; off > 0; off >>= 1) {
            b.lx = fminf(b.lx, __shfl_xor_sync(0xffffffffu, b.lx, off));
            b.ly = fminf(b.ly, __shfl_xor_sync(0xffffffffu, b.ly, off));
            b.lz = fminf(b.lz, __shfl_xor_sync(0xffffffffu, b.lz, off));
            b.hx = fmaxf(b.hx, __shfl_xor_sync(0xffffffffu, b.hx, off));
            b.hy = fmaxf(b.hy, __shfl_xor_sync(0xffffffffu, b.hy, off));
            b.hz = fmaxf(b.hz, __shfl_xor_sync(0xffffffffu, b.hz, off));
        }
        if ((threadIdx.x & 31) != 0) return;
    } else if (!valid) {
        return;
    }
    atomicMin(&sb[0], float_to_ordered(b.lx));
    atomicMin(&sb[1], float_to_ordered(b.ly));
    atomicMin(&sb[2], float_to_ordered(b.lz));
    atomicMax(&sb[3], float_to_ordered(b.hx));
    atomicMax(&sb[4], float_to_ordered(b.hy));
    atomicMax(&sb[5], float_to_ordered(b.hz));
}

__global__ void k_init_bounds(int* scene, int nseg) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nseg * 6) return;
    // +inf as ordered int for mins; -inf (0xFF800000 -> ordered 0x807FFFFF) for maxes
    scene[i] = (i % 6) < 3 ? 0x7F800000 : (int)0x807FFFFF;
}

// PT:913-920 expandBits: bit i of the 10-bit input moves to bit 3i.
__device__ __forceinline__ uint32_t expand_bits(uint32_t v) {
    uint32_t r = 0;
#pragma unroll
    for (int i = 0; i < 10; i++) r |= ((v >> i) & 1u) << (3 * i);
    return r;
}

// PT:922-925 quantize: (value - min) / (max - min) * 1023, then the host's
// float -> unsigned conversion (x86-64: truncation through a 64-bit integer,
// NaN -> 0, low 32 bits kept).
__device__ __forceinline__ uint32_t quantize(float value, float lo, float hi) {
    float normalized = __fdiv_rn(__fsub_rn(value, lo), __fsub_rn(hi, lo));
    float scaled = __fmul_rn(normalized, 1023.0f);
    if (scaled != scaled) return 0u;
    long long v = __float2ll_rz(scaled);
    return (uint32_t)v;
}

__global__ void k_morton(const float4* __restrict__ centroids, int n, const int* __restrict__ scene,
                         uint32_t* __restrict__ codes, int32_t* __restrict__ values) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 c = centroids[i];
    const int* sb = scene + 6 * __float_as_int(c.w);
    float lx = ordered_to_float(sb[0]), ly = ordered_to_float(sb[1]), lz = ordered_to_float(sb[2]);
    float hx = ordered_to_float(sb[3]), hy = ordered_to_float(sb[4]), hz = ordered_to_float(sb[5]);
    uint32_t x = expand_bits(quantize(c.x, lx, hx));
    uint32_t y = expand_bits(quantize(c.y, ly, hy));
    uint32_t z = expand_bits(quantize(c.z, lz, hz));
    codes[i] = x | y << 1 | z << 2;  // PT:934
    if (values) values[i] = i;
}

// Segment id of the primitive each sorted slot holds (the key of the final stable pass).
__global__ void k_segment_keys(const float4* __restrict__ centroids, const int32_t* __restrict__ order, int n,
                               uint32_t* __restrict__ keys) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) keys[k] = (uint32_t)__float_as_int(centroids[order[k]].w);
}

// ---------------------------------------------------------------------------
// Onesweep radix sort (Adinets & Merrill, "Onesweep: A Faster Least
// Significant Digit Radix Sort for GPUs", 2022): one histogram pass over the
// keys for all digit positions, then one kernel per digit position that ranks
// a tile, resolves its global digit offsets by decoupled look-back, and
// scatters. Ranking inside a tile is stable (warp match + running per-warp
// digit counts), so the sort is stable.
// ---------------------------------------------------------------------------
__global__ void k_radix_histogram(const uint32_t* __restrict__ keys, int n, int passes, uint32_t* __restrict__ hist) {
    __shared__ uint32_t h[4][kRadix];
    for (int i = threadIdx.x; i < 4 * kRadix; i += blockDim.x) (&h[0][0])[i] = 0;
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t k = keys[i];
        for (int p = 0; p < passes; p++) atomicAdd(&h[p][(k >> (p * kRadixBits)) & (kRadix - 1)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * kRadix; i += blockDim.x) {
        uint32_t v = (&h[0][0])[i];
        if (v) atomicAdd(&hist[i], v);
    }
}

__global__ void k_radix_scan(uint32_t* __restrict__ hist, int passes) {
    // one block of 256 threads per digit position: exclusive scan in place
    __shared__ uint32_t s[kRadix];
    int p = blockIdx.x;
    if (p >= passes) return;
    uint32_t v = hist[p * kRadix + threadIdx.x];
    s[threadIdx.x] = v;
    __syncthreads();
    for (int off = 1; off < kRadix; off <<= 1) {
        uint32_t t = threadIdx.x >= (unsigned)off ? s[threadIdx.x - off] : 0u;
        __syncthreads();
        s[threadIdx.x] += t;
        __syncthreads();
    }
    hist[p * kRadix + threadIdx.x] = s[threadIdx.x] - v;
}

__global__ void __launch_bounds__(kSortThreads) k_onesweep(const uint32_t* __restrict__ keys_in, const int32_t* __restrict__ vals_in,
                                 uint32_t* __restrict__ keys_out, int32_t* __restrict__ vals_out, int n, int shift,
                                 const uint32_t* __restrict__ digit_offsets, uint32_t* status, int* tile_counter,
                                 int* error) {
    __shared__ uint32_t warp_hist[kSortWarps][kRadix];
    __shared__ uint32_t digit_base[kRadix];
    __shared__ int tile_s;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) tile_s = atomicAdd(tile_counter, 1);
    for (int i = threadIdx.x; i < kSortWarps * kRadix; i += kSortThreads) (&warp_hist[0][0])[i] = 0;
    __syncthreads();
    const int tile = tile_s;
    const long long base = (long long)tile * kTile + (long long)warp * 32 * kSortItems;

    uint32_t key[kSortItems];
    int32_t val[kSortItems];
    uint32_t rank[kSortItems];
    const uint32_t lanemask_lt = (1u << lane) - 1u;
#pragma unroll
    for (int j = 0; j < kSortItems; j++) {
        long long idx = base + j * 32 + lane;
        bool valid = idx < n;
        key[j] = valid ? keys_in[idx] : 0xFFFFFFFFu;
        val[j] = valid ? vals_in[idx] : 0;
        uint32_t d = valid ? ((key[j] >> shift) & (kRadix - 1)) : (kRadix + lane);
        uint32_t peers = __match_any_sync(0xffffffffu, d);
        uint32_t prior = valid ? warp_hist[warp][d] : 0u;
        __syncwarp();
        rank[j] = prior + __popc(peers & lanemask_lt);
        int leader = __ffs(peers) - 1;
        if (valid && lane == leader) warp_hist[warp][d] = prior + __popc(peers);
        __syncwarp();
    }
    __syncthreads();

    // exclusive scan over warps for each digit; tile total per digit
    const int d = threadIdx.x;  // kSortThreads == kRadix
    uint32_t total = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; w++) {
        uint32_t t = warp_hist[w][d];
        warp_hist[w][d] = total;
        total += t;
    }
    // decoupled look-back over the preceding tiles for this digit
    volatile uint32_t* vstatus = status;
    uint32_t exclusive = 0;
    if (tile == 0) {
        vstatus[d] = kFlagInc | total;
    } else {
        vstatus[(long long)tile * kRadix + d] = kFlagAgg | total;
        int pred = tile - 1;
        long long spins = 0;
        while (pred >= 0) {
            uint32_t s = vstatus[(long long)pred * kRadix + d];
            uint32_t flag = s & ~kCountMask;
            if (flag == 0u) {
                if (++spins > kSpinLimit) {
                    atomicOr(error, MC_DEVERR_TIMEOUT);
                    break;
                }
                continue;
            }
            exclusive += s & kCountMask;
            if (flag == kFlagInc) break;
            pred--;
        }
        __threadfence();
        vstatus[(long long)tile * kRadix + d] = kFlagInc | (exclusive + total);
    }
    digit_base[d] = digit_offsets[d] + exclusive;
    __syncthreads();

#pragma unroll
    for (int j = 0; j < kSortItems; j++) {
        long long idx = base + j * 32 + lane;
        if (idx < n) {
            uint32_t dd = (key[j] >> shift) & (kRadix - 1);
            uint32_t dst = digit_base[dd] + warp_hist[warp][dd] + rank[j];
            if (dst < (uint32_t)n) {
                keys_out[dst] = key[j];
                vals_out[dst] = val[j];
            } else {
                atomicOr(error, MC_DEVERR_INPUT);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Karras 2012 hierarchy (PT:1337-1447), per segment.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int delta(const uint32_t* __restrict__ codes, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    uint32_t ci = codes[i], cj = codes[j];
    if (ci == cj) return 32 + __clz((unsigned int)(i ^ j));
    return __clz(ci ^ cj);
}

// Internal node g (global) of segment s works on the segment's codes with the
// local index g - intOff. Child references are global: internal child c ->
// intOff + c; leaf child k -> ~(primOff + k). parents: internal nodes at
// [0, NI), leaves at [NI, NI + N); value (global parent << 1) | side, -1 at roots.
__global__ void k_karras(const uint32_t* __restrict__ codes, const Seg* __restrict__ seg, int nseg, int NI,
                         float4* __restrict__ nodes, int32_t* __restrict__ parents, mc_bvh_node* __restrict__ ref_internal,
                         mc_bvh_node* __restrict__ ref_leaves, int2* __restrict__ ranges) {
    int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= NI) return;
    const int s = seg_of_internal(seg, nseg, g);
    const Seg& S = seg[s];
    const int n = S.ns + S.nt;
    const int idx = g - S.intOff;
    const uint32_t* c = codes + S.primOff;
    int d = (delta(c, n, idx, idx + 1) - delta(c, n, idx, idx - 1)) >= 0 ? 1 : -1;
    int deltaMin = delta(c, n, idx, idx - d);
    int lmax = 2;
    while (delta(c, n, idx, idx + lmax * d) > deltaMin) lmax *= 2;
    int l = 0;
    for (int t = lmax / 2; t >= 1; t /= 2)
        if (delta(c, n, idx, idx + (l + t) * d) > deltaMin) l += t;
    int jdx = idx + l * d;
    int first = min(idx, jdx);
    int last = max(idx, jdx);
    int common = delta(c, n, first, last);
    int split = first;
    int step = last - first;
    do {
        step = (step + 1) >> 1;
        int ns = split + step;
        if (ns < last && delta(c, n, first, ns) > common) split = ns;
    } while (step > 1);

    bool leftLeaf = (split == first);
    bool rightLeaf = (split + 1 == last);
    ranges[g] = make_int2(first, last);
    int leftRef = leftLeaf ? ~(S.primOff + split) : (S.intOff + split);
    int rightRef = rightLeaf ? ~(S.primOff + split + 1) : (S.intOff + split + 1);
    nodes[(long long)g * 4 + 3] = make_float4(__int_as_float(leftRef), __int_as_float(rightRef), 0.f, 0.f);
    parents[leftLeaf ? (NI + S.primOff + split) : (S.intOff + split)] = (g << 1) | 0;
    parents[rightLeaf ? (NI + S.primOff + split + 1) : (S.intOff + split + 1)] = (g << 1) | 1;
    if (idx == 0) parents[g] = -1;
    if (ref_internal) {  // single-scene builds only: the reference's node arrays
        mc_bvh_node& r = ref_internal[idx];
        r.left = split;
        r.right = split + 1;
        r.left_is_leaf = leftLeaf;
        r.right_is_leaf = rightLeaf;
        r.is_leaf = 0;
        r.prim = -1;
        if (idx == 0) r.parent = -1;
        if (leftLeaf) ref_leaves[split].parent = idx; else ref_internal[split].parent = idx;
        if (rightLeaf) ref_leaves[split + 1].parent = idx; else ref_internal[split + 1].parent = idx;
    }
}

__device__ __forceinline__ void store_child_box(float4* nodes, int node, int side, const Box& b) {
    float* f = reinterpret_cast<float*>(nodes + (long long)node * 4);
    int o = side ? 6 : 0;
    __stcg(f + o + 0, b.lx);
    __stcg(f + o + 1, b.ly);
    __stcg(f + o + 2, b.lz);
    __stcg(f + o + 3, b.hx);
    __stcg(f + o + 4, b.hy);
    __stcg(f + o + 5, b.hz);
}

__device__ __forceinline__ Box load_child_box(const float4* nodes, int node, int side) {
    const float* f = reinterpret_cast<const float*>(nodes + (long long)node * 4);
    int o = side ? 6 : 0;
    Box b;
    b.lx = __ldcg(f + o + 0);
    b.ly = __ldcg(f + o + 1);
    b.lz = __ldcg(f + o + 2);
    b.hx = __ldcg(f + o + 3);
    b.hy = __ldcg(f + o + 4);
    b.hz = __ldcg(f + o + 5);
    return b;
}

__device__ __forceinline__ mc_aabb to_aabb(const Box& b) {
    mc_aabb m;
    m.lo = mc_vec3{b.lx, b.ly, b.lz};
    m.hi = mc_vec3{b.hx, b.hy, b.hz};
    m.pad0 = 0.f;
    m.pad1 = 0.f;
    return m;
}

// Leaves + refit (buildLeavesKernel PT:1388-1396 and refitBoundsKernel
// PT:1398-1415): leaf k writes its primitive record and its box into the
// parent's slot; the second thread to arrive at a node merges the two slots
// and continues upwards. order[k] is the global (batch) primitive index.
__global__ void k_leaves_refit(const int32_t* __restrict__ order, const mc_aabb* __restrict__ bounds_ref, int N, int NI,
                               const Seg* __restrict__ seg, int nseg, float4* __restrict__ nodes,
                               float4* __restrict__ prims, const int32_t* __restrict__ parents, int* __restrict__ counters,
                               int32_t* __restrict__ ids_out, int32_t* __restrict__ types_out,
                               mc_bvh_node* __restrict__ ref_internal, mc_bvh_node* __restrict__ ref_leaves,
                               mc_aabb* __restrict__ root_boxes, int* __restrict__ err) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= N) return;
    int src = order[k];
    int s = seg_of_prim(seg, nseg, src);
    const Seg& S = seg[s];
    int local = src - S.primOff;
    int type = local < S.ns ? 0 : 1;
    int id = local < S.ns ? local : local - S.ns;
    float4 r0, r1, r2;
    if (type == 1) {
        const mc_triangle_hot t = S.hot[id];
        r0 = make_float4(t.v0.x, t.v0.y, t.v0.z, t.v1.x);
        r1 = make_float4(t.v1.y, t.v1.z, t.v2.x, t.v2.y);
        r2 = make_float4(t.v2.z, __int_as_float(id), __int_as_float(1), 0.f);
    } else {
        const mc_sphere& sp = S.sph[id];
        r0 = make_float4(sp.center.x, sp.center.y, sp.center.z, sp.center1.x);
        r1 = make_float4(sp.center1.y, sp.center1.z, sp.radius, sp.is_moving ? 1.f : 0.f);
        r2 = make_float4(0.f, __int_as_float(id), __int_as_float(0), 0.f);
    }
    prims[(long long)k * 3 + 0] = r0;
    prims[(long long)k * 3 + 1] = r1;
    prims[(long long)k * 3 + 2] = r2;
    if (ids_out) ids_out[k] = id;
    if (types_out) types_out[k] = type;
    mc_aabb a = bounds_ref[src];
    Box b = {a.lo.x, a.lo.y, a.lo.z, a.hi.x, a.hi.y, a.hi.z};
    if (ref_leaves) {
        mc_bvh_node& r = ref_leaves[k];
        r.bounds = a;
        r.prim = id;
        r.is_leaf = 1;
        r.left = -1;
        r.right = -1;
        r.left_is_leaf = 0;
        r.right_is_leaf = 0;
    }
    if (S.ns + S.nt == 1) {
        root_boxes[s] = a;
        return;
    }
    int p = parents[NI + k];
    if (p < 0) {
        atomicOr(err, MC_DEVERR_INPUT);  // every leaf of a Karras tree over n >= 2 keys has a parent
        return;
    }
    for (int level = 0; p >= 0; level++) {
        int node = p >> 1, side = p & 1;
        if (node >= NI || level > 2 * MC_STACK_CAPACITY) {
            atomicOr(err, MC_DEVERR_INPUT);
            return;
        }
        store_child_box(nodes, node, side, b);
        __threadfence();
        int old = atomicAdd(&counters[node], 1);
        if (old == 0) return;
        __threadfence();
        Box other = load_child_box(nodes, node, side ^ 1);
        b = side ? merge_box(other, b) : merge_box(b, other);
        if (ref_internal) ref_internal[node - S.intOff].bounds = to_aabb(b);
        p = parents[node];
        if (p < 0) root_boxes[s] = to_aabb(b);
    }
}

// The single-primitive tree: one node whose left child is leaf 0 and whose
// right child is an empty box (the reference needs n >= 2).
__global__ void k_single_root(float4* nodes, const mc_aabb* bounds) {
    mc_aabb a = bounds[0];
    nodes[0] = make_float4(a.lo.x, a.lo.y, a.lo.z, a.hi.x);
    nodes[1] = make_float4(a.hi.y, a.hi.z, INFINITY, INFINITY);
    nodes[2] = make_float4(INFINITY, -INFINITY, -INFINITY, -INFINITY);
    nodes[3] = make_float4(__int_as_float(~0), __int_as_float(~0), 0.f, 0.f);
}

// ---------------------------------------------------------------------------
// 4-wide collapse.
// Leaf rank = position of the leaf in the reference's traversal order with
// every box overlapping (stepTraversal PT:1276-1321): at a node its leaf
// children are tested first (left, then right), then its internal children are
// descended left first. Walking up from a leaf, each ancestor adds the number
// of leaves emitted before the branch that holds it. Ranks are made global by
// the segment's first primitive index.
// ---------------------------------------------------------------------------
__global__ void k_leaf_rank(const float4* __restrict__ nodes, const int32_t* __restrict__ parents,
                            const int2* __restrict__ ranges, const Seg* __restrict__ seg, int nseg, int N, int NI,
                            int* __restrict__ rank, int* err) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= N) return;
    const Seg& S = seg[seg_of_prim(seg, nseg, k)];
    if (S.ns + S.nt == 1) {
        rank[k] = k;
        return;
    }
    int r = 0;
    int p = parents[NI + k];
    for (int level = 0; p >= 0; level++) {
        int node = p >> 1, side = p & 1;
        if (node >= NI || level > 2 * MC_STACK_CAPACITY) {
            atomicOr(err, MC_DEVERR_INPUT);
            return;
        }
        float4 d = nodes[(long long)node * 4 + 3];
        int lref = __float_as_int(d.x), rref = __float_as_int(d.y);
        bool lLeaf = lref < 0, rLeaf = rref < 0;
        if (side == 0) {
            if (rLeaf && !lLeaf) r += 1;           // the right leaf is tested before the left subtree
        } else {
            if (lLeaf) r += 1;                      // the left leaf comes first
            else if (!rLeaf) r += ranges[lref].y - ranges[lref].x + 1;  // the whole left subtree comes first
        }
        p = parents[node];
    }
    rank[k] = S.primOff + r;
}

// Depth parity of internal nodes: wide nodes are the binary nodes at even depth
// of their tree. Roots record their wide id per segment.
__global__ void k_wide_select(const int32_t* __restrict__ parents, const Seg* __restrict__ seg, int nseg, int NI,
                              int* __restrict__ wideId, int* counter, int* __restrict__ wideRoot) {
    int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= NI) return;
    int depth = 0;
    int p = parents[g];
    while (p >= 0 && depth <= 4 * MC_STACK_CAPACITY) {
        depth++;
        p = parents[p >> 1];
    }
    if (depth & 1) {
        wideId[g] = -1;
    } else {
        int id = atomicAdd(counter, 1);
        wideId[g] = id;
        if (parents[g] < 0) wideRoot[seg_of_internal(seg, nseg, g)] = id;
    }
}

// Surface-area-greedy collapse: a wide node rooted at binary node B starts
// with B's two children and repeatedly opens its internal slot of largest
// surface area (ties: lowest slot) until it holds four slots or only leaves.
// Every slot is a node of the binary tree, so every box stays exact.
struct WideSlots {
    int n;
    int ref[4];   // binary child reference (internal index, or ~leaf)
    int par[4];   // binary node whose record holds the slot's box
    int side[4];
};

__device__ __forceinline__ float slot_area(const float4* nodes, int par, int side) {
    const float* f = reinterpret_cast<const float*>(nodes + (long long)par * 4) + (side ? 6 : 0);
    float dx = f[3] - f[0], dy = f[4] - f[1], dz = f[5] - f[2];
    return dx * dy + dy * dz + dz * dx;
}

__device__ void greedy_slots(const float4* nodes, int B, WideSlots& w) {
    float4 d = nodes[(long long)B * 4 + 3];
    w.n = 2;
    w.ref[0] = __float_as_int(d.x); w.par[0] = B; w.side[0] = 0;
    w.ref[1] = __float_as_int(d.y); w.par[1] = B; w.side[1] = 1;
    while (w.n < 4) {
        int best = -1;
        float bestA = -1.0f;
        for (int j = 0; j < w.n; j++) {
            if (w.ref[j] < 0) continue;
            float a = slot_area(nodes, w.par[j], w.side[j]);
            if (a > bestA) {
                bestA = a;
                best = j;
            }
        }
        if (best < 0) break;
        const int X = w.ref[best];
        float4 dx = nodes[(long long)X * 4 + 3];
        w.ref[best] = __float_as_int(dx.x); w.par[best] = X; w.side[best] = 0;
        w.ref[w.n] = __float_as_int(dx.y); w.par[w.n] = X; w.side[w.n] = 1;
        w.n++;
    }
}

// Wide id i for the i-th scene root.
__global__ void k_scatter_ids(const int* __restrict__ roots, int n, int* __restrict__ wideId) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) wideId[roots[i]] = i;
}

// One level of the collapse, in three steps so that wide ids follow the
// frontier's order (the same layout on every build: breadth first, the
// internal children of a wide node consecutive, in slot order).
// Count: every wide node of the frontier picks its slots, keeps its internal
// ones in slot order and adds their number to its tile's total (tile = kBlock
// frontier entries, one block; warpSum: kBlock / 32 entries).
__device__ __forceinline__ void wide_count_tile(const float4* nodes, const int* frontier, int n, int capacity,
                                                const int* wideId, int* rootOf, int4* internal, int* blockTotals, int* err,
                                                int tile, int* warpSum) {
    const int i = tile * kBlock + threadIdx.x;
    int nInt = 0;
    if (i < n) {
        const int B = frontier[i];
        const int w = wideId[B];
        int r[4] = {-1, -1, -1, -1};
        if (w < 0 || w >= capacity) {
            atomicOr(err, MC_DEVERR_INPUT);
        } else {
            rootOf[w] = B;
            WideSlots s;
            greedy_slots(nodes, B, s);
            for (int j = 0; j < s.n; j++)
                if (s.ref[j] >= 0) r[nInt++] = s.ref[j];
        }
        internal[i] = make_int4(r[0], r[1], r[2], r[3]);
    }
    int v = nInt;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) warpSum[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int k = 0; k < kBlock / 32; k++) t += warpSum[k];
        blockTotals[tile] = t;
    }
    __syncthreads();  // warpSum is reused by the block's next tile
}

__global__ void __launch_bounds__(kBlock) k_wide_level_count(const float4* __restrict__ nodes,
                                                             const int* __restrict__ frontier, int n, int capacity,
                                                             const int* __restrict__ wideId, int* __restrict__ rootOf,
                                                             int4* __restrict__ internal, int* __restrict__ blockTotals,
                                                             int* err) {
    __shared__ int warpSum[kBlock / 32];
    wide_count_tile(nodes, frontier, n, capacity, wideId, rootOf, internal, blockTotals, err, blockIdx.x, warpSum);
}

// Scan: exclusive prefix of `count` ints in place by one block (a multiple of
// 32 threads, at most 1024; warpSums: 32 entries); the total goes to *total.
__device__ __forceinline__ void scan_ints_block(int* v, int count, int* total, int* warpSums, int& carry) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < count; base += blockDim.x) {
        const int t = base + threadIdx.x;
        const int c = t < count ? v[t] : 0;
        int x = c;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warpSums[wid] = x;
        __syncthreads();
        if (wid == 0) {
            int s = lane < (int)(blockDim.x >> 5) ? warpSums[lane] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, s, o);
                if (lane >= o) s += y;
            }
            warpSums[lane] = s;
        }
        __syncthreads();
        const int before = carry + (wid > 0 ? warpSums[wid - 1] : 0) + x - c;
        if (t < count) v[t] = before;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = before + c;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

__global__ void __launch_bounds__(1024) k_wide_level_scan(int* blockTotals, int blocks, int* total) {
    __shared__ int warpSums[32];
    __shared__ int carry;
    scan_ints_block(blockTotals, blocks, total, warpSums, carry);
}

// Write: the internal children of frontier node i take wide ids idBase + o,
// o = (internal children of the nodes before i), and the same places of the
// next frontier.
__device__ __forceinline__ void wide_write_tile(const int4* internal, int n, const int* blockFirst, int idBase,
                                                int capacity, int* next, int* wideId, int* err, int tile, int* warpSum) {
    const int i = tile * kBlock + threadIdx.x;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int4 r = make_int4(-1, -1, -1, -1);
    if (i < n) r = internal[i];
    const int nInt = (r.x >= 0) + (r.y >= 0) + (r.z >= 0) + (r.w >= 0);
    int x = nInt;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warpSum[wid] = x;
    __syncthreads();
    int off = blockFirst[tile] + x - nInt;
    for (int k = 0; k < wid; k++) off += warpSum[k];
    const int refs[4] = {r.x, r.y, r.z, r.w};
    for (int k = 0; k < nInt; k++) {
        if (off + k >= capacity || idBase + off + k >= capacity) {
            atomicOr(err, MC_DEVERR_INPUT);
            break;
        }
        wideId[refs[k]] = idBase + off + k;
        next[off + k] = refs[k];
    }
    __syncthreads();  // warpSum is reused by the block's next tile
}

__global__ void __launch_bounds__(kBlock) k_wide_level_write(const int4* __restrict__ internal, int n,
                                                             const int* __restrict__ blockFirst, int idBase,
                                                             int capacity, int* __restrict__ next,
                                                             int* __restrict__ wideId, int* err) {
    __shared__ int warpSum[kBlock / 32];
    wide_write_tile(internal, n, blockFirst, idBase, capacity, next, wideId, err, blockIdx.x, warpSum);
}

// Every level of the collapse in one cooperative launch: the three steps of
// a level as loops over the same tiles, a grid-wide barrier after each; all
// blocks read the level's total from the same place after a barrier, so they
// run the same levels. Ends when a level adds no internal node, after
// maxLevels + 1 levels, or when the wide ids would pass the node count (error).
struct WideLevels {
    const float4* nodes;
    int* front[2];
    int nseg, capacity, maxLevels;
    int* wideId;
    int* rootOf;
    int4* internal;
    int* blockTotals;
    int* total;
    int* out;  // [0] levels, [1] wide nodes, [2] last frontier size, [3] 1 when the ids would pass capacity
    int* err;
};

__global__ void __launch_bounds__(kBlock) k_wide_levels(WideLevels a) {
    cooperative_groups::grid_group grid = cooperative_groups::this_grid();
    __shared__ int warpSum[32];
    __shared__ int carry;
    int n = a.nseg, idBase = a.nseg, cur = 0, levels = 0;
    bool bad = false;
    while (n > 0 && levels <= a.maxLevels) {
        const int* front = cur ? a.front[1] : a.front[0];
        int* next = cur ? a.front[0] : a.front[1];
        const int tiles = (n + kBlock - 1) / kBlock;
        for (int t = blockIdx.x; t < tiles; t += gridDim.x)
            wide_count_tile(a.nodes, front, n, a.capacity, a.wideId, a.rootOf, a.internal, a.blockTotals, a.err, t,
                            warpSum);
        grid.sync();
        if (blockIdx.x == 0) scan_ints_block(a.blockTotals, tiles, a.total, warpSum, carry);
        grid.sync();
        for (int t = blockIdx.x; t < tiles; t += gridDim.x)
            wide_write_tile(a.internal, n, a.blockTotals, idBase, a.capacity, next, a.wideId, a.err, t, warpSum);
        grid.sync();
        const int m = *a.total;  // written by block 0 before the last barrier
        if (m < 0 || (long long)idBase + m > a.capacity) {
            bad = true;
            break;
        }
        idBase += m;
        n = m;
        cur = 1 - cur;
        levels++;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.out[0] = levels;
        a.out[1] = idBase;
        a.out[2] = n;
        a.out[3] = bad ? 1 : 0;
    }
}

// Writes every wide node of the greedy collapse from its slots.
__global__ void k_wide_fill_greedy(const float4* __restrict__ nodes, const int* __restrict__ rootOf,
                                   const int* __restrict__ wideId, const int* __restrict__ rank, int count,
                                   float4* __restrict__ wide) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= count) return;
    WideSlots s;
    greedy_slots(nodes, rootOf[id], s);
    float lo[3][4], hi[3][4];
    int ref[4];
    for (int c = 0; c < 4; c++) {
        if (c < s.n) {
            const float* f = reinterpret_cast<const float*>(nodes + (long long)s.par[c] * 4) + (s.side[c] ? 6 : 0);
            lo[0][c] = f[0]; lo[1][c] = f[1]; lo[2][c] = f[2];
            hi[0][c] = f[3]; hi[1][c] = f[4]; hi[2][c] = f[5];
            ref[c] = s.ref[c] < 0 ? ~rank[~s.ref[c]] : wideId[s.ref[c]];
        } else {
            lo[0][c] = lo[1][c] = lo[2][c] = INFINITY;
            hi[0][c] = hi[1][c] = hi[2][c] = -INFINITY;
            ref[c] = MC_WIDE_EMPTY;
        }
    }
    float4* w = wide + (long long)id * 8;
    w[0] = make_float4(lo[0][0], lo[0][1], lo[0][2], lo[0][3]);
    w[1] = make_float4(lo[1][0], lo[1][1], lo[1][2], lo[1][3]);
    w[2] = make_float4(lo[2][0], lo[2][1], lo[2][2], lo[2][3]);
    w[3] = make_float4(hi[0][0], hi[0][1], hi[0][2], hi[0][3]);
    w[4] = make_float4(hi[1][0], hi[1][1], hi[1][2], hi[1][3]);
    w[5] = make_float4(hi[2][0], hi[2][1], hi[2][2], hi[2][3]);
    w[6] = make_float4(__int_as_float(ref[0]), __int_as_float(ref[1]), __int_as_float(ref[2]), __int_as_float(ref[3]));
    w[7] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// Quantised 4-wide node (64 bytes), from an exact one (128 bytes):
//   float4 0: frame origin (x, y, z) = the union's low corner; w = the three
//             scale exponents (e + 128, one byte per axis)
//   float4 1: lo.x, lo.y, lo.z, hi.x of the 4 children, one byte per child
//   float4 2: hi.y, hi.z of the 4 children; two spare words
//   float4 3: the 4 child references (as in the exact layout)
// A plane decodes as origin + q * 2^e. q is chosen so that this decode, which
// is exact up to one rounding of the sum (q * 2^e is exact), lies at or
// outside the exact plane: low planes round down, high planes round up.
// Exponents stay >= -100 so no decode term is subnormal.
__device__ __forceinline__ float q_decode(float origin, int q, int e) {
    return origin + (float)q * __int_as_float((e + 127) << 23);
}

__global__ void k_quantize_wide(const float4* __restrict__ exact, int count, float4* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float4* n = exact + (size_t)i * 8;
    const float4 lx = n[0], ly = n[1], lz = n[2], hx = n[3], hy = n[4], hz = n[5], rf = n[6];
    const float lo[3][4] = {{lx.x, lx.y, lx.z, lx.w}, {ly.x, ly.y, ly.z, ly.w}, {lz.x, lz.y, lz.z, lz.w}};
    const float hi[3][4] = {{hx.x, hx.y, hx.z, hx.w}, {hy.x, hy.y, hy.z, hy.w}, {hz.x, hz.y, hz.z, hz.w}};
    const int ref[4] = {__float_as_int(rf.x), __float_as_int(rf.y), __float_as_int(rf.z), __float_as_int(rf.w)};
    float origin[3];
    int ex[3];
    unsigned qlo[3][4], qhi[3][4];
    for (int a = 0; a < 3; a++) {
        float ulo = INFINITY, uhi = -INFINITY;
        for (int c = 0; c < 4; c++) {
            if (ref[c] == MC_WIDE_EMPTY) continue;
            ulo = fminf(ulo, lo[a][c]);
            uhi = fmaxf(uhi, hi[a][c]);
        }
        if (!(ulo <= uhi)) { ulo = 0.f; uhi = 0.f; }
        origin[a] = ulo;
        int e = -100;
        const double ext = (double)uhi - (double)ulo;
        if (ext > 0.0) e = max(-100, (int)ceil(log2(ext / 255.0)));
        while (e < 127 && q_decode(ulo, 255, e) < uhi) e++;
        ex[a] = e;
        for (int c = 0; c < 4; c++) {
            if (ref[c] == MC_WIDE_EMPTY) {
                qlo[a][c] = 255;  // empty: low above high
                qhi[a][c] = 0;
                continue;
            }
            const double s = ldexp(1.0, e);
            int ql = (int)floor(((double)lo[a][c] - (double)ulo) / s);
            ql = min(255, max(0, ql));
            while (ql > 0 && q_decode(ulo, ql, e) > lo[a][c]) ql--;
            int qh = (int)ceil(((double)hi[a][c] - (double)ulo) / s);
            qh = min(255, max(0, qh));
            while (qh < 255 && q_decode(ulo, qh, e) < hi[a][c]) qh++;
            qlo[a][c] = (unsigned)ql;
            qhi[a][c] = (unsigned)qh;
        }
    }
    auto pack = [](const unsigned* v) { return v[0] | (v[1] << 8) | (v[2] << 16) | (v[3] << 24); };
    const unsigned exps = (unsigned)(ex[0] + 128) | ((unsigned)(ex[1] + 128) << 8) | ((unsigned)(ex[2] + 128) << 16);
    float4* o = out + (size_t)i * 4;
    o[0] = make_float4(origin[0], origin[1], origin[2], __int_as_float((int)exps));
    o[1] = make_float4(__int_as_float((int)pack(qlo[0])), __int_as_float((int)pack(qlo[1])),
                       __int_as_float((int)pack(qlo[2])), __int_as_float((int)pack(qhi[0])));
    o[2] = make_float4(__int_as_float((int)pack(qhi[1])), __int_as_float((int)pack(qhi[2])), 0.f, 0.f);
    o[3] = rf;
}

__device__ __forceinline__ void child_slot_box(const float4* nodes, int node, int side, float* b) {
    const float* f = reinterpret_cast<const float*>(nodes + (long long)node * 4);
    int o = side ? 6 : 0;
#pragma unroll
    for (int j = 0; j < 6; j++) b[j] = f[o + j];
}

// One wide node per selected binary node: its children, with each internal
// child replaced by that child's two children. Boxes are copied exactly.
__global__ void k_wide_fill(const float4* __restrict__ nodes, const int* __restrict__ wideId, const int* __restrict__ rank,
                            int NI, float4* __restrict__ wide) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= NI) return;
    int id = wideId[i];
    if (id < 0) return;
    float lo[3][4], hi[3][4];
    int ref[4];
    int c = 0;
    float4 d = nodes[(long long)i * 4 + 3];
    int kids[2] = {__float_as_int(d.x), __float_as_int(d.y)};
    for (int side = 0; side < 2; side++) {
        int kref = kids[side];
        if (kref < 0) {
            float b[6];
            child_slot_box(nodes, i, side, b);
            lo[0][c] = b[0]; lo[1][c] = b[1]; lo[2][c] = b[2];
            hi[0][c] = b[3]; hi[1][c] = b[4]; hi[2][c] = b[5];
            ref[c++] = ~rank[~kref];
        } else {
            float4 dd = nodes[(long long)kref * 4 + 3];
            int gk[2] = {__float_as_int(dd.x), __float_as_int(dd.y)};
            for (int gs = 0; gs < 2; gs++) {
                float b[6];
                child_slot_box(nodes, kref, gs, b);
                lo[0][c] = b[0]; lo[1][c] = b[1]; lo[2][c] = b[2];
                hi[0][c] = b[3]; hi[1][c] = b[4]; hi[2][c] = b[5];
                int g = gk[gs];
                ref[c++] = g < 0 ? ~rank[~g] : wideId[g];
            }
        }
    }
    for (; c < 4; c++) {
        lo[0][c] = lo[1][c] = lo[2][c] = INFINITY;
        hi[0][c] = hi[1][c] = hi[2][c] = -INFINITY;
        ref[c] = MC_WIDE_EMPTY;
    }
    float4* w = wide + (long long)id * 8;
    w[0] = make_float4(lo[0][0], lo[0][1], lo[0][2], lo[0][3]);
    w[1] = make_float4(lo[1][0], lo[1][1], lo[1][2], lo[1][3]);
    w[2] = make_float4(lo[2][0], lo[2][1], lo[2][2], lo[2][3]);
    w[3] = make_float4(hi[0][0], hi[0][1], hi[0][2], hi[0][3]);
    w[4] = make_float4(hi[1][0], hi[1][1], hi[1][2], hi[1][3]);
    w[5] = make_float4(hi[2][0], hi[2][1], hi[2][2], hi[2][3]);
    w[6] = make_float4(__int_as_float(ref[0]), __int_as_float(ref[1]), __int_as_float(ref[2]), __int_as_float(ref[3]));
    w[7] = make_float4(0.f, 0.f, 0.f, 0.f);
}

__global__ void k_reorder_prims(const float4* __restrict__ src, const int* __restrict__ rank, int n, float4* __restrict__ dst) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    int r = rank[k];
    dst[(long long)r * 3 + 0] = src[(long long)k * 3 + 0];
    dst[(long long)r * 3 + 1] = src[(long long)k * 3 + 1];
    dst[(long long)r * 3 + 2] = src[(long long)k * 3 + 2];
}

__global__ void k_leaf_depth(const int32_t* __restrict__ parents, int N, int NI, int* depth) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= N) return;
    int dcount = 0;
    int p = parents[NI + k];
    while (p >= 0) {
        p = parents[p >> 1];
        dcount++;
        if (dcount > 4 * MC_STACK_CAPACITY) break;
    }
    atomicMax(depth, dcount);
}

// dst[i] = src[idx[i]] for a caller-supplied order; out-of-range entries are
// flagged (and read as 0) instead of being dereferenced.
__global__ void k_gather_u32(const uint32_t* __restrict__ src, const int32_t* __restrict__ idx, int n, uint32_t* __restrict__ dst,
                             int* err) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int j = idx[i];
    if (j < 0 || j >= n) {
        atomicOr(err, MC_DEVERR_INPUT);
        dst[i] = 0u;
        return;
    }
    dst[i] = src[j];
}

// A caller-supplied order must be a permutation that sorts the codes.
__global__ void k_check_order(const int32_t* __restrict__ order, const uint32_t* __restrict__ sorted, int n, int* seen, int* err) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    int j = order[k];
    if (j < 0 || j >= n) {
        atomicOr(err, MC_DEVERR_INPUT);
        return;
    }
    if (atomicExch(&seen[j], 1) != 0) atomicOr(err, MC_DEVERR_INPUT);
    if (k > 0 && sorted[k] < sorted[k - 1]) atomicOr(err, MC_DEVERR_INPUT);
}

int grid_for(long long n, int block) { return (int)std::max(1ll, (n + block - 1) / block); }

}  // namespace

namespace mc {

// Sorts (keys, values) pairs of n entries stably by the low key_bits bits.
// keys/vals are sorted in place; alt_keys/alt_vals are scratch of n entries.
mc_status radix_sort_pairs(mc_context* ctx, uint32_t* keys, int32_t* vals, uint32_t* alt_keys, int32_t* alt_vals, int n,
                           int key_bits) {
    if (n <= 1) return MC_OK;
    int passes = (key_bits + kRadixBits - 1) / kRadixBits;
    if (passes < 1 || passes > 4) return set_error(MC_ERR_INVALID, "radix sort: key_bits must be in [1, 32]");
    long long tiles = (n + kTile - 1) / kTile;
    size_t statusBytes = (size_t)tiles * kRadix * sizeof(uint32_t);
    size_t histBytes = 4 * kRadix * sizeof(uint32_t);
    mc_status st = devbuf_reserve(ctx->scratch[6], histBytes + 16 * sizeof(int) + (size_t)passes * statusBytes);
    if (st != MC_OK) return st;
    char* base = (char*)ctx->scratch[6].ptr;
    uint32_t* hist = (uint32_t*)base;
    int* tileCounters = (int*)(base + histBytes);
    uint32_t* status = (uint32_t*)(base + histBytes + 16 * sizeof(int));
    MC_CUDA(cudaMemsetAsync(base, 0, histBytes + 16 * sizeof(int) + (size_t)passes * statusBytes, ctx->stream));
    int hblocks = std::min(grid_for(n, 256), ctx->sm_count * 4);
    k_radix_histogram<<<hblocks, 256, 0, ctx->stream>>>(keys, n, passes, hist);
    k_radix_scan<<<passes, kRadix, 0, ctx->stream>>>(hist, passes);
    uint32_t* kin = keys; int32_t* vin = vals; uint32_t* kout = alt_keys; int32_t* vout = alt_vals;
    for (int p = 0; p < passes; p++) {
        k_onesweep<<<(int)tiles, kSortThreads, 0, ctx->stream>>>(kin, vin, kout, vout, n, p * kRadixBits, hist + p * kRadix,
                                                                 status + (size_t)p * tiles * kRadix, tileCounters + p,
                                                                 ctx->d_error);
        std::swap(kin, kout);
        std::swap(vin, vout);
    }
    if (kin != keys) {
        MC_CUDA(cudaMemcpyAsync(keys, kin, (size_t)n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, ctx->stream));
        MC_CUDA(cudaMemcpyAsync(vals, vin, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToDevice, ctx->stream));
    }
    MC_CUDA(cudaGetLastError());
    return MC_OK;
}

}  // namespace mc

// ---------------------------------------------------------------------------
// Radix sort over a fixed scratch array (no device allocation).
// Byte layout of the array, every part 256-byte aligned:
//   [alternate keys: MAX u32][alternate values: MAX i32]
//   [histograms: 4 x 256 u32][tile counters: 64 i32][status: 4 x tiles x 256 u32]
// ---------------------------------------------------------------------------
namespace {
constexpr size_t kStaticPairs = MC_SORT_STATIC_MAX_PAIRS;
constexpr size_t kStaticTiles = (kStaticPairs + kTile - 1) / kTile;
constexpr size_t kStaticValsOff = kStaticPairs * sizeof(uint32_t);
constexpr size_t kStaticHistOff = kStaticValsOff + kStaticPairs * sizeof(int32_t);
constexpr size_t kStaticCounterOff = kStaticHistOff + 4 * kRadix * sizeof(uint32_t);
constexpr size_t kStaticStatusOff = kStaticCounterOff + 64 * sizeof(int);
constexpr size_t kStaticBytes = kStaticStatusOff + 4 * kStaticTiles * kRadix * sizeof(uint32_t);
static_assert(kStaticValsOff % 256 == 0 && kStaticHistOff % 256 == 0 && kStaticCounterOff % 256 == 0 &&
                  kStaticStatusOff % 256 == 0,
              "scratch parts must stay 256-byte aligned");
constexpr int kStaticMaxDevices = 64;
}  // namespace

static __device__ __align__(256) unsigned char g_sort_scratch[kStaticBytes];

namespace mc {
namespace {

std::mutex g_static_mu;
void* g_static_scratch[kStaticMaxDevices] = {};

// Address of this device's scratch array; looked up once per device with the
// device current. Also loads the sort kernels, so later calls load nothing.
mc_status static_sort_scratch(int device, char** out) {
    if (device < 0 || device >= kStaticMaxDevices) return set_error(MC_ERR_INVALID, "static sort: device %d out of range", device);
    std::lock_guard<std::mutex> lock(g_static_mu);
    if (!g_static_scratch[device]) {
        int cur = -1;
        cudaError_t e = cudaGetDevice(&cur);
        if (e != cudaSuccess) return cuda_error((int)e, "cudaGetDevice", __FILE__, __LINE__);
        if (cur != device && (e = cudaSetDevice(device)) != cudaSuccess) return cuda_error((int)e, "cudaSetDevice", __FILE__, __LINE__);
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_sort_scratch);
        cudaFuncAttributes fa;
        if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_radix_histogram);
        if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_radix_scan);
        if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_onesweep);
        if (cur != device) cudaSetDevice(cur);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return cuda_error((int)e, "static sort set-up (cudaGetSymbolAddress)", __FILE__, __LINE__);
        }
        if (!p) return set_error(MC_ERR_CUDA, "static sort: null scratch address");
        g_static_scratch[device] = p;
    }
    *out = (char*)g_static_scratch[device];
    return MC_OK;
}

}  // namespace

mc_status radix_sort_pairs_static(mc_context* ctx, uint32_t* keys, int32_t* vals, int n, int key_bits) {
    char* base = nullptr;
    mc_status st = static_sort_scratch(ctx->device, &base);
    if (st != MC_OK) return st;
    if (n <= 1) return MC_OK;
    const int passes = (key_bits + kRadixBits - 1) / kRadixBits;
    const long long tiles = (n + kTile - 1) / kTile;
    uint32_t* altKeys = (uint32_t*)base;
    int32_t* altVals = (int32_t*)(base + kStaticValsOff);
    uint32_t* hist = (uint32_t*)(base + kStaticHistOff);
    int* tileCounters = (int*)(base + kStaticCounterOff);
    uint32_t* status = (uint32_t*)(base + kStaticStatusOff);
    // histograms, tile counters and the status words of the used passes start at zero
    const size_t zeroBytes = (kStaticStatusOff - kStaticHistOff) + (size_t)passes * tiles * kRadix * sizeof(uint32_t);
    MC_CUDA(cudaMemsetAsync(base + kStaticHistOff, 0, zeroBytes, ctx->stream));
    int hblocks = std::min(grid_for(n, 256), ctx->sm_count * 4);
    k_radix_histogram<<<hblocks, 256, 0, ctx->stream>>>(keys, n, passes, hist);
    k_radix_scan<<<passes, kRadix, 0, ctx->stream>>>(hist, passes);
    uint32_t* kin = keys; int32_t* vin = vals; uint32_t* kout = altKeys; int32_t* vout = altVals;
    for (int p = 0; p < passes; p++) {
        k_onesweep<<<(int)tiles, kSortThreads, 0, ctx->stream>>>(kin, vin, kout, vout, n, p * kRadixBits, hist + p * kRadix,
                                                                 status + (size_t)p * tiles * kRadix, tileCounters + p,
                                                                 ctx->d_error);
        std::swap(kin, kout);
        std::swap(vin, vout);
    }
    if (kin != keys) {
        MC_CUDA(cudaMemcpyAsync(keys, kin, (size_t)n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, ctx->stream));
        MC_CUDA(cudaMemcpyAsync(vals, vin, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToDevice, ctx->stream));
    }
    MC_CUDA(cudaGetLastError());
    return MC_OK;
}

// Build buffers come from the device's stream-ordered pool (pool_alloc): they
// are taken and returned in stream order, without a device-wide wait.
template <class T>
static bool palloc(mc_context* ctx, T** p, size_t bytes) {
    void* v = nullptr;
    const bool ok = pool_alloc(ctx, &v, bytes) == MC_OK;
    *p = (T*)v;
    return ok;
}

mc_status bvh_depth(mc_bvh* bvh) {
    if (bvh->depth >= 0) return MC_OK;
    if (bvh->n == 1) {
        bvh->depth = 1;
        return MC_OK;
    }
    mc_context* ctx = bvh->ctx;
    int* d;
    if (!palloc(ctx, &d, sizeof(int))) return MC_ERR_OOM;
    MC_CUDA(cudaMemsetAsync(d, 0, sizeof(int), ctx->stream));
    k_leaf_depth<<<grid_for(bvh->n, kBlock), kBlock, 0, ctx->stream>>>(bvh->parents, bvh->n, bvh->ni, d);
    int h = 0;
    MC_CUDA(cudaMemcpyAsync(&h, d, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    MC_CUDA(cudaStreamSynchronize(ctx->stream));
    pool_free(ctx, d);
    bvh->depth = h;
    return MC_OK;
}

static mc_status check_scene(const mc_scene_view* s) {
    if (!s) return set_error(MC_ERR_INVALID, "null scene");
    if (s->sphere_count < 0 || s->triangle_count < 0) return set_error(MC_ERR_INVALID, "negative primitive count");
    long long n = (long long)s->sphere_count + s->triangle_count;
    if (n == 0) return set_error(MC_ERR_INVALID, "the scene has no primitives");
    if (n >= (1ll << 30)) return set_error(MC_ERR_INVALID, "too many primitives (limit 2^30 - 1)");
    if (s->sphere_count > 0 && !s->spheres) return set_error(MC_ERR_INVALID, "null sphere array");
    if (s->triangle_count > 0 && !s->tri_hot) return set_error(MC_ERR_INVALID, "null triangle array");
    return MC_OK;
}

static mc_status flags_now(mc_context* ctx, int* flags) {
    MC_CUDA(cudaMemcpyAsync(flags, ctx->d_error, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    MC_CUDA(cudaStreamSynchronize(ctx->stream));
    return MC_OK;
}

// Uploads the segment table of the given scenes to ctx->scratch[7] (after the
// per-segment bounds words) and returns the device pointers.
static mc_status upload_segments(mc_context* ctx, const mc_scene_view* views, int nseg, std::vector<Seg>& segs, Seg** dSeg,
                                 int** dBounds, mc_aabb** dRootBoxes, int** dWideRoot) {
    segs.resize(nseg);
    int prim = 0;
    for (int s = 0; s < nseg; s++) {
        segs[s].sph = views[s].spheres;
        segs[s].hot = views[s].tri_hot;
        segs[s].ns = views[s].sphere_count;
        segs[s].nt = views[s].triangle_count;
        segs[s].primOff = prim;
        segs[s].intOff = prim - s;
        prim += segs[s].ns + segs[s].nt;
    }
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    size_t bBytes = al((size_t)nseg * 6 * sizeof(int));
    size_t sBytes = al((size_t)nseg * sizeof(Seg));
    size_t rBytes = al((size_t)nseg * sizeof(mc_aabb));
    size_t wBytes = al((size_t)nseg * sizeof(int));
    mc_status st = devbuf_reserve(ctx->scratch[7], bBytes + sBytes + rBytes + wBytes);
    if (st != MC_OK) return st;
    char* base = (char*)ctx->scratch[7].ptr;
    *dBounds = (int*)base;
    *dSeg = (Seg*)(base + bBytes);
    *dRootBoxes = (mc_aabb*)(base + bBytes + sBytes);
    *dWideRoot = (int*)(base + bBytes + sBytes + rBytes);
    MC_CUDA(cudaMemcpyAsync(*dSeg, segs.data(), (size_t)nseg * sizeof(Seg), cudaMemcpyHostToDevice, ctx->stream));
    k_init_bounds<<<grid_for(nseg * 6, kBlock), kBlock, 0, ctx->stream>>>(*dBounds, nseg);
    return MC_OK;
}

// 4-wide collapse of a finished binary build (Karras ranges in ctx->scratch[1]).
// ---------------------------------------------------------------------------
// The traversal tree of the wide layouts: PLOC (parallel locally-ordered
// clustering, Meister and Bittner 2018) over the same Morton-sorted leaves.
// Each round, every cluster finds the neighbour within kPlocRadius positions
// (same scene) whose merged box has the least surface area; mutual nearest
// neighbours merge into a new internal node, which takes the lower position,
// and the clusters are compacted in order. The round's globally closest pair
// (ties: lower positions) is always mutual, so every scene with two or more
// clusters loses at least one per round. The result replaces the LBVH as
// the binary tree the 4-wide collapse reads: on this renderer's scenes it
// needs about 40 % fewer wide-node visits per ray (large triangles, such as a
// ground plane or an area light, are spread over the whole LBVH by their
// centroids; clustering by merged area keeps them near the root). The LBVH
// stays for the binary layout, the exported reference nodes, and the leaf
// ranks: leaves keep their reference-rank slots, so the tie rule, and with
// it every hit, is the same with either tree.
// ---------------------------------------------------------------------------
constexpr int kPlocRadius = 8;  // 8, 16, 32 measured within 1 % of each other; 8 builds fastest
constexpr int kPlocBlock = 256;
constexpr int kScanItems = 4;  // items per thread of the block scans

// cluster k <- leaf k: reference ~k, box (lo.w = scene)
__global__ void k_ploc_init(const int32_t* __restrict__ order, const mc_aabb* __restrict__ bounds, const Seg* __restrict__ seg,
                            int nseg, int N, int* __restrict__ cref, float4* __restrict__ cbox) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
        const mc_aabb b = bounds[order[k]];
        const int s = seg_of_prim(seg, nseg, k);
        cref[k] = ~k;
        cbox[2 * (long long)k] = make_float4(b.lo.x, b.lo.y, b.lo.z, __int_as_float(s));
        cbox[2 * (long long)k + 1] = make_float4(b.hi.x, b.hi.y, b.hi.z, 0.f);
    }
}

__device__ __forceinline__ float merged_area(float4 alo, float4 ahi, float4 blo, float4 bhi) {
    const float dx = fmaxf(ahi.x, bhi.x) - fminf(alo.x, blo.x);
    const float dy = fmaxf(ahi.y, bhi.y) - fminf(alo.y, blo.y);
    const float dz = fmaxf(ahi.z, bhi.z) - fminf(alo.z, blo.z);
    return dx * dy + dy * dz + dz * dx;
}

// nn[i] = the position j != i, |i - j| <= kPlocRadius, same scene, of least
// merged area (ties: the lower j); -1 when no cluster of its scene is near.
// One block of kPlocBlock threads takes the positions b0 .. b0 + kPlocBlock - 1
// through a shared window (sLo / sHi: kPlocBlock + 2 kPlocRadius entries).
// Plain loads: the persistent rounds read what other blocks wrote earlier in
// the same launch.
__device__ __forceinline__ void ploc_nn_tile(const float4* cbox, int n, int b0, int* nn, float4* sLo, float4* sHi) {
    for (int t = threadIdx.x; t < kPlocBlock + 2 * kPlocRadius; t += blockDim.x) {
        const int g = b0 - kPlocRadius + t;
        if (g >= 0 && g < n) {
            sLo[t] = cbox[2 * (long long)g];
            sHi[t] = cbox[2 * (long long)g + 1];
        } else {
            sLo[t] = make_float4(INFINITY, INFINITY, INFINITY, __int_as_float(-1));
            sHi[t] = make_float4(-INFINITY, -INFINITY, -INFINITY, 0.f);
        }
    }
    __syncthreads();
    const int i = b0 + threadIdx.x;
    if (i < n) {
        const int me = threadIdx.x + kPlocRadius;
        const float4 lo = sLo[me], hi = sHi[me];
        const int s = __float_as_int(lo.w);
        float best = INFINITY;
        int bj = -1;
        for (int o = -kPlocRadius; o <= kPlocRadius; o++) {
            const int j = i + o;
            if (o == 0 || j < 0 || j >= n) continue;
            const float4 l2 = sLo[me + o];
            if (__float_as_int(l2.w) != s) continue;
            const float a = merged_area(lo, hi, l2, sHi[me + o]);
            if (a < best) {
                best = a;
                bj = j;
            }
        }
        nn[i] = bj;
    }
    __syncthreads();  // the window is refilled by the block's next tile
}

__global__ void __launch_bounds__(kPlocBlock) k_ploc_nn(const float4* __restrict__ cbox, const int* __restrict__ nPtr,
                                                         int* __restrict__ nn) {
    __shared__ float4 sLo[kPlocBlock + 2 * kPlocRadius], sHi[kPlocBlock + 2 * kPlocRadius];
    const int n = *nPtr;
    const int b0 = blockIdx.x * kPlocBlock;
    if (b0 >= n) return;
    ploc_nn_tile(cbox, n, b0, nn, sLo, sHi);
}

// (merge, alive) per cluster: a mutual pair merges at its lower position and
// the higher one disappears; every other cluster stays.
__device__ __forceinline__ int2 ploc_flag(const int* nn, int i) {
    const int j = nn[i];
    const bool mutual = j >= 0 && nn[j] == i;
    return make_int2(mutual && i < j ? 1 : 0, (!mutual || i < j) ? 1 : 0);
}

__global__ void k_ploc_flags(const int* __restrict__ nn, const int* __restrict__ nPtr, int2* __restrict__ flags) {
    const int n = *nPtr;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) flags[i] = ploc_flag(nn, i);
}

// Exclusive scan of int2 values: per tile of kPlocBlock * kScanItems items
// (one block of kPlocBlock threads; warpSum: kPlocBlock / 32 entries), then
// the tile sums (one block), then the offsets.
__device__ __forceinline__ void scan2_tile(const int2* in, int n, int tile, int2* out, int2* sums, int2* warpSum) {
    const long long base = ((long long)tile * kPlocBlock + threadIdx.x) * kScanItems;
    int2 v[kScanItems];
    int2 acc = make_int2(0, 0);
#pragma unroll
    for (int q = 0; q < kScanItems; q++) {
        const long long g = base + q;
        const int2 x = g < n ? in[g] : make_int2(0, 0);
        v[q] = acc;
        acc.x += x.x;
        acc.y += x.y;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int2 incl = acc;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int yx = __shfl_up_sync(0xffffffffu, incl.x, o), yy = __shfl_up_sync(0xffffffffu, incl.y, o);
        if (lane >= o) {
            incl.x += yx;
            incl.y += yy;
        }
    }
    if (lane == 31) warpSum[warp] = incl;
    __syncthreads();
    int2 before = make_int2(incl.x - acc.x, incl.y - acc.y);
    for (int w = 0; w < warp; w++) {
        before.x += warpSum[w].x;
        before.y += warpSum[w].y;
    }
#pragma unroll
    for (int q = 0; q < kScanItems; q++) {
        const long long g = base + q;
        if (g < n) out[g] = make_int2(before.x + v[q].x, before.y + v[q].y);
    }
    if (threadIdx.x == kPlocBlock - 1) sums[tile] = make_int2(before.x + acc.x, before.y + acc.y);
    __syncthreads();  // warpSum is reused by the block's next tile
}

__global__ void __launch_bounds__(kPlocBlock) k_scan2_blocks(const int2* __restrict__ in, const int* __restrict__ nPtr,
                                                              int2* __restrict__ out, int2* __restrict__ sums) {
    __shared__ int2 warpSum[kPlocBlock / 32];
    scan2_tile(in, *nPtr, blockIdx.x, out, sums, warpSum);
}

// Exclusive scan of the nb tile sums in place by one block (any multiple of
// 32 threads; warpSum: blockDim.x / 32 entries); the grand total goes to *total.
__device__ __forceinline__ void scan2_sums_block(int2* sums, int nb, int2* total, int2* warpSum, int2& carry) {
    if (threadIdx.x == 0) carry = make_int2(0, 0);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int start = 0; start < nb; start += blockDim.x) {
        const int i = start + threadIdx.x;
        const int2 x = i < nb ? sums[i] : make_int2(0, 0);
        int2 incl = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int yx = __shfl_up_sync(0xffffffffu, incl.x, o), yy = __shfl_up_sync(0xffffffffu, incl.y, o);
            if (lane >= o) {
                incl.x += yx;
                incl.y += yy;
            }
        }
        if (lane == 31) warpSum[warp] = incl;
        __syncthreads();
        int2 before = make_int2(carry.x + incl.x - x.x, carry.y + incl.y - x.y);
        for (int w = 0; w < warp; w++) {
            before.x += warpSum[w].x;
            before.y += warpSum[w].y;
        }
        if (i < nb) sums[i] = before;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = make_int2(before.x + x.x, before.y + x.y);
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

__global__ void __launch_bounds__(1024) k_scan2_sums(int2* __restrict__ sums, int nb, int2* __restrict__ total) {
    __shared__ int2 warpSum[32];
    __shared__ int2 carry;
    scan2_sums_block(sums, nb, total, warpSum, carry);
}

__global__ void k_scan2_add(int2* __restrict__ out, const int* __restrict__ nPtr, const int2* __restrict__ sums) {
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= *nPtr) return;
    const int2 off = sums[g / (kPlocBlock * kScanItems)];
    const int2 v = out[g];
    out[g] = make_int2(v.x + off.x, v.y + off.y);
}

// Writes the round's new internal nodes (binary layout: left box, right box,
// references) and the compacted clusters. pi: cluster i's (node, cluster)
// places among the round's merges and survivors.
__device__ __forceinline__ void ploc_emit_one(const int* cref, const float4* cbox, const int* nn, int2 f, int2 pi, int i,
                                              int nodeBase, int nodeCap, float4* nodes, int* crefOut, float4* cboxOut,
                                              int* err) {
    if (!f.y) return;
    const int p = pi.y;
    const float4 alo = cbox[2 * (long long)i], ahi = cbox[2 * (long long)i + 1];
    if (f.x) {
        const int j = nn[i];
        const int node = nodeBase + pi.x;
        if (node >= nodeCap) {
            atomicOr(err, MC_DEVERR_INPUT);
            return;
        }
        const float4 blo = cbox[2 * (long long)j], bhi = cbox[2 * (long long)j + 1];
        float4* o = nodes + (long long)node * 4;
        o[0] = make_float4(alo.x, alo.y, alo.z, ahi.x);
        o[1] = make_float4(ahi.y, ahi.z, blo.x, blo.y);
        o[2] = make_float4(blo.z, bhi.x, bhi.y, bhi.z);
        o[3] = make_float4(__int_as_float(cref[i]), __int_as_float(cref[j]), 0.f, 0.f);
        crefOut[p] = node;
        cboxOut[2 * (long long)p] = make_float4(fminf(alo.x, blo.x), fminf(alo.y, blo.y), fminf(alo.z, blo.z), alo.w);
        cboxOut[2 * (long long)p + 1] = make_float4(fmaxf(ahi.x, bhi.x), fmaxf(ahi.y, bhi.y), fmaxf(ahi.z, bhi.z), 0.f);
    } else {
        crefOut[p] = cref[i];
        cboxOut[2 * (long long)p] = alo;
        cboxOut[2 * (long long)p + 1] = ahi;
    }
}

__global__ void k_ploc_emit(const int* __restrict__ cref, const float4* __restrict__ cbox, const int* __restrict__ nn,
                            const int2* __restrict__ flags, const int2* __restrict__ pos, const int* __restrict__ state,
                            int nodeCap, float4* __restrict__ nodes, int* __restrict__ crefOut, float4* __restrict__ cboxOut,
                            int* __restrict__ err) {
    const int n = state[0], nodeBase = state[1];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        ploc_emit_one(cref, cbox, nn, flags[i], pos[i], i, nodeBase, nodeCap, nodes, crefOut, cboxOut, err);
}

// End of a round: the cluster count and the next node id move on; a round
// without a merge while a scene still has two clusters is an error (it
// cannot happen: the closest pair is mutual).
__global__ void k_ploc_advance(const int2* __restrict__ total, int* __restrict__ state, int nseg, int* __restrict__ err) {
    const int2 t = *total;
    if (t.x == 0) {
        if (state[0] > nseg) atomicOr(err, MC_DEVERR_INPUT);
        return;
    }
    state[1] += t.x;
    state[0] = t.y;
}

// Every clustering round in one cooperative launch. A round's phases (nearest
// neighbours, merge flags, tile scans, the scan of the tile sums by block 0,
// emit) take the same tiles as the per-phase launches above, as grid-stride
// loops, with a grid-wide barrier after each; every block reads the round's
// totals from the same place after a barrier, so all blocks run the same
// rounds and reach the same barriers, and the tree is the per-phase launches'
// to the bit. The loop ends when every scene is one cluster, after maxRounds
// rounds (error), or when a round merges nothing (error: the globally closest
// pair is always mutual).
struct PlocRounds {
    int* cref[2];
    float4* cbox[2];
    int* nn;
    int2* flags;
    int2* pos;
    int2* sums;
    int2* total;
    int* state;  // out: [0] clusters left, [1] internal nodes written, [2] buffer of the last clusters, [3] rounds
    float4* nodes;
    int nodeCap, nseg, N, maxRounds;
    int* err;
};

__global__ void __launch_bounds__(kPlocBlock) k_ploc_rounds(PlocRounds a) {
    cooperative_groups::grid_group grid = cooperative_groups::this_grid();
    __shared__ float4 sLo[kPlocBlock + 2 * kPlocRadius], sHi[kPlocBlock + 2 * kPlocRadius];
    __shared__ int2 warpSum[kPlocBlock / 32];
    __shared__ int2 carry;
    const int per = kPlocBlock * kScanItems;
    const long long stride = (long long)gridDim.x * blockDim.x;
    int n = a.N, nodeBase = 0, cur = 0, round = 0;
    bool failed = false;
    while (n > a.nseg) {
        if (round >= a.maxRounds) {
            failed = true;
            break;
        }
        const int* cref = cur ? a.cref[1] : a.cref[0];
        const float4* cbox = cur ? a.cbox[1] : a.cbox[0];
        int* crefOut = cur ? a.cref[0] : a.cref[1];
        float4* cboxOut = cur ? a.cbox[0] : a.cbox[1];
        for (int b0 = blockIdx.x * kPlocBlock; b0 < n; b0 += gridDim.x * kPlocBlock)
            ploc_nn_tile(cbox, n, b0, a.nn, sLo, sHi);
        grid.sync();
        for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
            a.flags[i] = ploc_flag(a.nn, (int)i);
        grid.sync();
        const int nb = (n + per - 1) / per;
        for (int t = blockIdx.x; t < nb; t += gridDim.x) scan2_tile(a.flags, n, t, a.pos, a.sums, warpSum);
        grid.sync();
        if (blockIdx.x == 0) scan2_sums_block(a.sums, nb, a.total, warpSum, carry);
        grid.sync();
        for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
            const int2 pi = a.pos[i], off = a.sums[i / per];
            ploc_emit_one(cref, cbox, a.nn, a.flags[i], make_int2(pi.x + off.x, pi.y + off.y), (int)i, nodeBase,
                          a.nodeCap, a.nodes, crefOut, cboxOut, a.err);
        }
        grid.sync();
        const int2 t = *a.total;  // written by block 0 before the last two barriers
        if (t.x == 0) {
            failed = true;
            break;
        }
        nodeBase += t.x;
        n = t.y;
        cur = 1 - cur;
        round++;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.state[0] = n;
        a.state[1] = nodeBase;
        a.state[2] = cur;
        a.state[3] = round;
        if (failed) atomicOr(a.err, MC_DEVERR_INPUT);
    }
}

// Builds the clustered tree into tree->nodes (NI internal nodes) and its
// scene roots; MC_ERR_UNSUPPORTED when a scene has fewer than two primitives
// (the caller keeps the LBVH then).
struct ClusterTree {
    float4* nodes = nullptr;
    std::vector<int> roots;
};

static mc_status build_ploc(mc_context* ctx, const mc_bvh* bvh, const Seg* dSeg, int nseg, const int32_t* order,
                            const mc_aabb* bounds, ClusterTree& tree, bool coop) {
    const int N = bvh->n, NI = bvh->ni;
    if (NI <= 0 || N < 2) return MC_ERR_UNSUPPORTED;
    const int per = kPlocBlock * kScanItems;
    const long long nbMax = (N + per - 1) / per;
    const size_t bytes = (size_t)NI * 64 + 2 * (size_t)N * 4 + 4 * (size_t)N * 16 + (size_t)N * 4 + 2 * (size_t)N * 8 +
                         (size_t)(nbMax + 1) * 8 + 32 + 16 * 16;  // + the 16-byte rounding of each part
    char* mem = nullptr;
    if (!palloc(ctx, &mem, bytes)) {
        cudaGetLastError();
        return set_error(MC_ERR_OOM, "mc_bvh_build: clustering scratch allocation failed");
    }
    char* p = mem;
    auto take = [&](size_t b) { char* r = p; p += (b + 15) & ~(size_t)15; return r; };
    tree.nodes = (float4*)take((size_t)NI * 64);
    int* cref[2] = {(int*)take((size_t)N * 4), (int*)take((size_t)N * 4)};
    float4* cbox[2] = {(float4*)take((size_t)N * 32), (float4*)take((size_t)N * 32)};
    int* nn = (int*)take((size_t)N * 4);
    int2* flags = (int2*)take((size_t)N * 8);
    int2* pos = (int2*)take((size_t)N * 8);
    int2* sums = (int2*)take((size_t)(nbMax + 1) * 8);
    int2* total = (int2*)take(32);  // the round's totals, then [2..3] as ints: clusters, next node id
    auto fail = [&](mc_status s) {
        pool_free(ctx, mem);
        tree.nodes = nullptr;
        return s;
    };
    const int loop = ctx->sm_count * 8;
    int* state = (int*)(total + 2);  // [0] clusters, [1] next node id
    k_ploc_init<<<std::min(grid_for(N, kBlock), loop), kBlock, 0, ctx->stream>>>(order, bounds, dSeg, nseg, N, cref[0], cbox[0]);
    const int h0[2] = {N, 0};
    if (cudaMemcpyAsync(state, h0, sizeof(h0), cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess)
        return fail(cuda_error(cudaGetLastError(), "mc_bvh_build (clustering)", __FILE__, __LINE__));
    int n = N, nodeBase = 0, cur = 0, rounds = 0;
    // every round in one cooperative launch where the device supports it
    int coopAttr = 0, perSm = 0;
    if (coop && cudaDeviceGetAttribute(&coopAttr, cudaDevAttrCooperativeLaunch, ctx->device) == cudaSuccess && coopAttr &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_ploc_rounds, kPlocBlock, 0) == cudaSuccess && perSm > 0) {
        PlocRounds pr;
        pr.cref[0] = cref[0]; pr.cref[1] = cref[1];
        pr.cbox[0] = cbox[0]; pr.cbox[1] = cbox[1];
        pr.nn = nn; pr.flags = flags; pr.pos = pos; pr.sums = sums; pr.total = total; pr.state = state;
        pr.nodes = tree.nodes;
        pr.nodeCap = NI; pr.nseg = nseg; pr.N = N; pr.maxRounds = 4096;
        pr.err = ctx->d_error;
        void* args[] = {&pr};
        const int grid = (int)std::min<long long>((long long)perSm * ctx->sm_count, (N + kPlocBlock - 1) / kPlocBlock);
        if (cudaLaunchCooperativeKernel((const void*)k_ploc_rounds, grid, kPlocBlock, args, 0, ctx->stream) ==
            cudaSuccess) {
            int h[4];
            if (cudaMemcpyAsync(h, state, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
                cudaStreamSynchronize(ctx->stream) != cudaSuccess)
                return fail(cuda_error(cudaGetLastError(), "mc_bvh_build (clustering)", __FILE__, __LINE__));
            int fl = 0;
            mc_status fs = flags_now(ctx, &fl);
            if (fs != MC_OK || fl) return fail(fs != MC_OK ? fs : status_from_device_flags(fl));
            n = h[0];
            nodeBase = h[1];
            cur = h[2];
            rounds = h[3];
        } else {
            cudaGetLastError();  // the per-phase launches below instead
        }
    }
    // otherwise rounds in batches between host checks; every launch reads the
    // cluster count from the device and is sized for the last count seen
    const int kBatch = 8;
    while (n > nseg) {
        if (rounds > 4096) return fail(set_error(MC_ERR_INVALID, "mc_bvh_build: clustering did not converge"));
        const int nb = (n + per - 1) / per;
        for (int r = 0; r < kBatch; r++, rounds++) {
            k_ploc_nn<<<(n + kPlocBlock - 1) / kPlocBlock, kPlocBlock, 0, ctx->stream>>>(cbox[cur], state, nn);
            k_ploc_flags<<<std::min(grid_for(n, kBlock), loop), kBlock, 0, ctx->stream>>>(nn, state, flags);
            k_scan2_blocks<<<nb, kPlocBlock, 0, ctx->stream>>>(flags, state, pos, sums);
            k_scan2_sums<<<1, 1024, 0, ctx->stream>>>(sums, nb, total);
            k_scan2_add<<<grid_for(n, kBlock), kBlock, 0, ctx->stream>>>(pos, state, sums);
            k_ploc_emit<<<std::min(grid_for(n, kBlock), loop), kBlock, 0, ctx->stream>>>(
                cref[cur], cbox[cur], nn, flags, pos, state, NI, tree.nodes, cref[1 - cur], cbox[1 - cur], ctx->d_error);
            k_ploc_advance<<<1, 1, 0, ctx->stream>>>(total, state, nseg, ctx->d_error);
            cur = 1 - cur;
        }
        int h[2];
        if (cudaMemcpyAsync(h, state, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
            cudaStreamSynchronize(ctx->stream) != cudaSuccess)
            return fail(cuda_error(cudaGetLastError(), "mc_bvh_build (clustering)", __FILE__, __LINE__));
        int fl = 0;
        mc_status fs = flags_now(ctx, &fl);
        if (fs != MC_OK || fl) return fail(fs != MC_OK ? fs : status_from_device_flags(fl));
        n = h[0];
        nodeBase = h[1];
    }
    tree.roots.assign((size_t)nseg, -1);
    if (cudaMemcpyAsync(tree.roots.data(), cref[cur], (size_t)nseg * 4, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
        cudaStreamSynchronize(ctx->stream) != cudaSuccess)
        return fail(cuda_error(cudaGetLastError(), "mc_bvh_build (clustering)", __FILE__, __LINE__));
    int flagsNow = 0;
    mc_status st = flags_now(ctx, &flagsNow);
    if (st != MC_OK || flagsNow) return fail(st != MC_OK ? st : status_from_device_flags(flagsNow));
    if (nodeBase != NI || n != nseg) return fail(set_error(MC_ERR_INVALID, "mc_bvh_build: clustering left %d clusters", n));
    for (int r : tree.roots)
        if (r < 0) return fail(MC_ERR_UNSUPPORTED);  // a scene of one primitive: keep the LBVH
    // the node block starts the allocation, so freeing it frees everything
    return MC_OK;
}

// The 4-wide collapse of a binary tree: `tree` (binary node layout, NI
// internal nodes) with scene roots `roots`; the LBVH when tree is null. A
// clustered tree whose greedy collapse would outgrow the traversal stack
// returns MC_ERR_UNSUPPORTED (the caller then collapses the LBVH, which has
// the depth-parity fallback).
static mc_status build_wide(mc_context* ctx, mc_bvh* bvh, const Seg* dSeg, int nseg, int* dWideRoot, bool coop,
                            const float4* tree = nullptr, const std::vector<int>* roots = nullptr) {
    const int N = bvh->n, NI = bvh->ni;
    const float4* bin = tree ? tree : (const float4*)bvh->nodes;
    mc_status st;
    if ((st = devbuf_reserve(ctx->scratch[2], (size_t)N * 4 + 16)) != MC_OK) return st;
    if ((st = devbuf_reserve(ctx->scratch[3], (size_t)N * 4 + 16)) != MC_OK) return st;
    if ((st = devbuf_reserve(ctx->scratch[5], (size_t)N * 4 + 16)) != MC_OK) return st;
    int* rank = (int*)ctx->scratch[2].ptr;
    int* wideId = (int*)ctx->scratch[3].ptr;
    int* counter = (int*)ctx->scratch[5].ptr;
    k_leaf_rank<<<grid_for(N, kBlock), kBlock, 0, ctx->stream>>>((const float4*)bvh->nodes, bvh->parents,
                                                                (const int2*)ctx->scratch[1].ptr, dSeg, nseg, N, NI, rank,
                                                                ctx->d_error);
    int count = 1;
    int* rootOf = nullptr;   // greedy collapse: binary root of each wide node
    bool greedy = false;
    if (NI > 0) {
        // surface-area-greedy collapse, level by level from the scene roots
        int* front[2] = {nullptr, nullptr};
        int* cnt = nullptr;  // [0]: next frontier size; [4..7]: the cooperative collapse's results
        int4* internal = nullptr;  // per frontier node: its internal slots
        int* blockTotals = nullptr;
        auto release = [&]() {
            pool_free(ctx, front[0]);
            pool_free(ctx, front[1]);
            pool_free(ctx, cnt);
            pool_free(ctx, internal);
            pool_free(ctx, blockTotals);
        };
        if (!palloc(ctx, &rootOf, (size_t)NI * sizeof(int)) ||
            !palloc(ctx, &front[0], (size_t)NI * sizeof(int)) ||
            !palloc(ctx, &front[1], (size_t)NI * sizeof(int)) || !palloc(ctx, &cnt, 8 * sizeof(int)) ||
            !palloc(ctx, &internal, (size_t)NI * sizeof(int4)) ||
            !palloc(ctx, &blockTotals, (size_t)(grid_for(NI, kBlock) + 1) * sizeof(int))) {
            cudaGetLastError();
            release();
            pool_free(ctx, rootOf);
            return set_error(MC_ERR_OOM, "mc_bvh_build: wide-collapse scratch allocation failed");
        }
        MC_CUDA(cudaMemsetAsync(wideId, 0xFF, (size_t)NI * sizeof(int), ctx->stream));
        const std::vector<int> rootList = roots ? *roots : std::vector<int>(bvh->bin_roots.begin(), bvh->bin_roots.end());
        MC_CUDA(cudaMemcpyAsync(front[0], rootList.data(), rootList.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
        k_scatter_ids<<<grid_for(nseg, kBlock), kBlock, 0, ctx->stream>>>(front[0], nseg, wideId);
        // wide ids 0..nseg-1 are the roots; each level's children follow in frontier order
        int levels = 0, cur = 0, n = nseg, idBase = nseg;
        // every level in one cooperative launch where the device supports it
        int coopAttr = 0, perSm = 0;
        if (coop && cudaDeviceGetAttribute(&coopAttr, cudaDevAttrCooperativeLaunch, ctx->device) == cudaSuccess && coopAttr &&
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_wide_levels, kBlock, 0) == cudaSuccess && perSm > 0) {
            WideLevels wl;
            wl.nodes = bin;
            wl.front[0] = front[0];
            wl.front[1] = front[1];
            wl.nseg = nseg;
            wl.capacity = NI;
            wl.maxLevels = 4 * MC_STACK_CAPACITY;
            wl.wideId = wideId;
            wl.rootOf = rootOf;
            wl.internal = internal;
            wl.blockTotals = blockTotals;
            wl.total = cnt;
            wl.out = cnt + 4;
            wl.err = ctx->d_error;
            void* args[] = {&wl};
            const int grid = std::max(1, std::min(perSm * ctx->sm_count, grid_for(NI, kBlock)));
            if (cudaLaunchCooperativeKernel((const void*)k_wide_levels, grid, kBlock, args, 0, ctx->stream) ==
                cudaSuccess) {
                int h[4];
                MC_CUDA(cudaMemcpyAsync(h, cnt + 4, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
                MC_CUDA(cudaStreamSynchronize(ctx->stream));
                if (h[3]) {
                    release();
                    pool_free(ctx, rootOf);
                    return set_error(MC_ERR_INVALID, "mc_bvh_build: the collapse found more nodes than internal nodes");
                }
                levels = h[0];
                idBase = h[1];
                n = h[2];
            } else {
                cudaGetLastError();  // the per-level launches below instead
            }
        }
        while (n > 0 && levels <= 4 * MC_STACK_CAPACITY) {
            const int blocks = grid_for(n, kBlock);
            k_wide_level_count<<<blocks, kBlock, 0, ctx->stream>>>(bin, front[cur], n, NI, wideId, rootOf, internal,
                                                                   blockTotals, ctx->d_error);
            k_wide_level_scan<<<1, 1024, 0, ctx->stream>>>(blockTotals, blocks, cnt);
            k_wide_level_write<<<blocks, kBlock, 0, ctx->stream>>>(internal, n, blockTotals, idBase, NI, front[1 - cur],
                                                                   wideId, ctx->d_error);
            MC_CUDA(cudaMemcpyAsync(&n, cnt, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
            MC_CUDA(cudaStreamSynchronize(ctx->stream));
            if (n < 0 || (long long)idBase + n > NI) {
                // more wide nodes than internal nodes: not a binary tree over these leaves
                release();
                pool_free(ctx, rootOf);
                return set_error(MC_ERR_INVALID, "mc_bvh_build: the collapse found %d nodes past %d", n, idBase);
            }
            idBase += n;
            cur = 1 - cur;
            levels++;
        }
        count = idBase;
        int flags = 0;
        if ((st = flags_now(ctx, &flags)) != MC_OK || flags) {
            release();
            pool_free(ctx, rootOf);
            return st != MC_OK ? st : status_from_device_flags(flags);
        }
        release();
        // a visit pushes at most 3 siblings: the traversal stack must hold 3 per level
        greedy = n == 0 && 3 * levels <= MC_STACK_CAPACITY;
        bvh->wide_levels = greedy ? levels : -1;
        if (!greedy && tree) {
            pool_free(ctx, rootOf);
            return MC_ERR_UNSUPPORTED;
        }
        if (!greedy) {
            pool_free(ctx, rootOf);
            rootOf = nullptr;
            MC_CUDA(cudaMemsetAsync(counter, 0, sizeof(int), ctx->stream));
            k_wide_select<<<grid_for(NI, kBlock), kBlock, 0, ctx->stream>>>(bvh->parents, dSeg, nseg, NI, wideId, counter,
                                                                           dWideRoot);
            MC_CUDA(cudaMemcpyAsync(&count, counter, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        }
    }
    int flags = 0;
    if ((st = flags_now(ctx, &flags)) != MC_OK || flags) {
        pool_free(ctx, rootOf);
        return st != MC_OK ? st : status_from_device_flags(flags);
    }
    if (!palloc(ctx, &bvh->wide_nodes, (size_t)count * 128) ||
        !palloc(ctx, &bvh->wide_prims, (size_t)N * 48)) {
        cudaGetLastError();
        pool_free(ctx, rootOf);
        return set_error(MC_ERR_OOM, "mc_bvh_build: wide-node allocation failed");
    }
    bvh->wide_roots.assign(nseg, 0);
    if (NI > 0 && greedy) {
        k_wide_fill_greedy<<<grid_for(count, kBlock), kBlock, 0, ctx->stream>>>(bin, rootOf, wideId,
                                                                              rank, count, (float4*)bvh->wide_nodes);
        for (int s = 0; s < nseg; s++) bvh->wide_roots[s] = s;
        MC_CUDA(cudaStreamSynchronize(ctx->stream));
        pool_free(ctx, rootOf);
    } else if (NI > 0) {
        k_wide_fill<<<grid_for(NI, kBlock), kBlock, 0, ctx->stream>>>((const float4*)bvh->nodes, wideId, rank, NI,
                                                                     (float4*)bvh->wide_nodes);
        MC_CUDA(cudaMemcpyAsync(bvh->wide_roots.data(), dWideRoot, (size_t)nseg * sizeof(int), cudaMemcpyDeviceToHost,
                                ctx->stream));
    } else {
        // one leaf under the root, three empty slots
        float inf = INFINITY;
        mc_aabb a;
        MC_CUDA(cudaMemcpyAsync(&a, ctx->scratch[0].ptr, sizeof(a), cudaMemcpyDeviceToHost, ctx->stream));
        MC_CUDA(cudaStreamSynchronize(ctx->stream));
        float h[32] = {a.lo.x, inf, inf, inf, a.lo.y, inf, inf, inf, a.lo.z, inf, inf, inf,
                       a.hi.x, -inf, -inf, -inf, a.hi.y, -inf, -inf, -inf, a.hi.z, -inf, -inf, -inf};
        int refs[4] = {~0, MC_WIDE_EMPTY, MC_WIDE_EMPTY, MC_WIDE_EMPTY};
        memcpy(&h[24], refs, sizeof(refs));
        h[28] = h[29] = h[30] = h[31] = 0.f;
        MC_CUDA(cudaMemcpyAsync(bvh->wide_nodes, h, sizeof(h), cudaMemcpyHostToDevice, ctx->stream));
    }
    k_reorder_prims<<<grid_for(N, kBlock), kBlock, 0, ctx->stream>>>((const float4*)bvh->prims, rank, N,
                                                                    (float4*)bvh->wide_prims);
    MC_CUDA(cudaGetLastError());
    MC_CUDA(cudaStreamSynchronize(ctx->stream));
    bvh->wide_count = count;
    bvh->layout = MC_BVH_LAYOUT_WIDE4;
    return MC_OK;
}

// Builds one BVH over nseg scenes (nseg == 1: a single scene). The reference's
// node arrays (keep_reference_nodes) and an injected permutation are single-scene only.
mc_status build_segments(mc_context* ctx, const mc_scene_view* views, int nseg, const mc_bvh_build_opts* opts, mc_bvh** out) {
    if (!ctx || !out || !views || nseg < 1) return set_error(MC_ERR_INVALID, "mc_bvh_build: null argument");
    *out = nullptr;
    long long total = 0;
    for (int s = 0; s < nseg; s++) {
        mc_status st = check_scene(&views[s]);
        if (st != MC_OK) return st;
        long long ns = (long long)views[s].sphere_count + views[s].triangle_count;
        if (nseg > 1 && ns < 2) return set_error(MC_ERR_INVALID, "mc_bvh_build_batch: every scene needs at least 2 primitives");
        total += ns;
    }
    if (total >= (1ll << 30)) return set_error(MC_ERR_INVALID, "too many primitives in the batch (limit 2^30 - 1)");
    mc_bvh_build_opts o = {};
    if (opts) o = *opts;
    if (o.layout != MC_BVH_LAYOUT_BINARY && o.layout != MC_BVH_LAYOUT_WIDE4 && o.layout != MC_BVH_LAYOUT_WIDE4Q)
        return set_error(MC_ERR_INVALID, "mc_bvh_build: unknown layout");
    if (nseg > 1 && (o.permutation || o.keep_reference_nodes))
        return set_error(MC_ERR_INVALID, "mc_bvh_build_batch: permutation and reference nodes are single-scene options");
    const int N = (int)total;
    const int NI = N - nseg;  // every scene of n_s >= 1 primitives has n_s - 1 internal nodes

    mc_bvh* bvh = new mc_bvh();
    bvh->ctx = ctx;
    bvh->device = ctx->device;
    bvh->n = N;
    bvh->ni = NI;
    bvh->ns = nseg == 1 ? views[0].sphere_count : 0;
    bvh->nt = nseg == 1 ? views[0].triangle_count : 0;
    bvh->nseg = nseg;
    bvh->layout = MC_BVH_LAYOUT_BINARY;
    auto fail = [&](mc_status s) { mc_bvh_free(bvh); return s; };

    long long nodesCount = std::max(1, NI);
    if (!palloc(ctx, &bvh->nodes, (size_t)nodesCount * 64) ||
        !palloc(ctx, &bvh->prims, (size_t)N * 48) ||
        !palloc(ctx, &bvh->codes, (size_t)N * 4) ||
        !palloc(ctx, &bvh->ids, (size_t)N * 4) ||
        !palloc(ctx, &bvh->types, (size_t)N * 4) ||
        !palloc(ctx, &bvh->parents, (size_t)(NI + N) * 4 + 8)) {
        cudaGetLastError();
        return fail(set_error(MC_ERR_OOM, "mc_bvh_build: device allocation failed (n=%d)", N));
    }
    if (o.keep_reference_nodes) {
        if (!palloc(ctx, &bvh->ref_internal, (size_t)nodesCount * sizeof(mc_bvh_node)) ||
            !palloc(ctx, &bvh->ref_leaves, (size_t)N * sizeof(mc_bvh_node))) {
            cudaGetLastError();
            return fail(set_error(MC_ERR_OOM, "mc_bvh_build: device allocation failed (reference nodes)"));
        }
        cudaMemsetAsync(bvh->ref_internal, 0, (size_t)nodesCount * sizeof(mc_bvh_node), ctx->stream);
        cudaMemsetAsync(bvh->ref_leaves, 0, (size_t)N * sizeof(mc_bvh_node), ctx->stream);
    }
    bvh->node_count = nodesCount;
    bvh->node_bytes = nodesCount * 64;

    // scratch: [0] primitive boxes, [1] centroids then Karras ranges, [2]/[3] sort buffers,
    // [4] order, [5] refit counters, [6] sort status, [7] segment table + bounds words
    mc_status st;
    if ((st = devbuf_reserve(ctx->scratch[0], (size_t)N * sizeof(mc_aabb))) != MC_OK) return fail(st);
    if ((st = devbuf_reserve(ctx->scratch[1], (size_t)N * sizeof(float4))) != MC_OK) return fail(st);
    if ((st = devbuf_reserve(ctx->scratch[2], (size_t)N * 4 + 16)) != MC_OK) return fail(st);
    if ((st = devbuf_reserve(ctx->scratch[3], (size_t)N * 4 + 16)) != MC_OK) return fail(st);
    if ((st = devbuf_reserve(ctx->scratch[4], (size_t)N * 4 + 16)) != MC_OK) return fail(st);
    if ((st = devbuf_reserve(ctx->scratch[5], (size_t)nodesCount * 4 + 16)) != MC_OK) return fail(st);
    std::vector<Seg> segs;
    Seg* dSeg;
    int* dBounds;
    mc_aabb* dRootBoxes;
    int* dWideRoot;
    if ((st = upload_segments(ctx, views, nseg, segs, &dSeg, &dBounds, &dRootBoxes, &dWideRoot)) != MC_OK) return fail(st);
    mc_aabb* boundsRef = (mc_aabb*)ctx->scratch[0].ptr;
    float4* centroids = (float4*)ctx->scratch[1].ptr;
    int32_t* order = (int32_t*)ctx->scratch[4].ptr;
    int* counters = (int*)ctx->scratch[5].ptr;

    if (cudaMemsetAsync(ctx->d_error, 0, sizeof(int), ctx->stream) != cudaSuccess)
        return fail(cuda_error(cudaGetLastError(), "memset", __FILE__, __LINE__));
    k_prim_bounds<<<grid_for(N, kBlock), kBlock, 0, ctx->stream>>>(dSeg, nseg, N, boundsRef, centroids, dBounds);
    k_morton<<<grid_for(N, kBlock), kBlock, 0, ctx->stream>>>(centroids, N, dBounds, bvh->codes, order);
    if (o.permutation) {
        // caller-provided order (e.g. the reference's std::sort order)
        if (cudaMemcpyAsync(order, o.permutation, (size_t)N * 4, cudaMemcpyDeviceToDevice, ctx->stream) != cudaSuccess)
            return fail(cuda_error(cudaGetLastError(), "permutation copy", __FILE__, __LINE__));
        uint32_t* tmp = (uint32_t*)ctx->scratch[2].ptr;
        if (cudaMemcpyAsync(tmp, bvh->codes, (size_t)N * 4, cudaMemcpyDeviceToDevice, ctx->stream) != cudaSuccess)
            return fail(cuda_error(cudaGetLastError(), "code copy", __FILE__, __LINE__));
        k_gather_u32<<<grid_for(N, kBlock), kBlock, 0, ctx->stream>>>(tmp, order, N, bvh->codes, ctx->d_error);
        int* seen = (int*)ctx->scratch[3].ptr;
        if (cudaMemsetAsync(seen, 0, (size_t)N * 4, ctx->stream) != cudaSuccess)
            return fail(cuda_error(cudaGetLastError(), "memset", __FILE__, __LINE__));
        k_check_order<<<grid_for(N, kBlock), kBlock, 0, ctx->stream>>>(order, bvh->codes, N, seen, ctx->d_error);
    } else {
        st = radix_sort_pairs(ctx, bvh->codes, order, (uint32_t*)ctx->scratch[2].ptr, (int32_t*)ctx->scratch[3].ptr, N, 30);
        if (st != MC_OK) return fail(st);
        if (nseg > 1) {
            // stable pass on the segment id: the order becomes (segment, code);
            // the codes follow through a copy in ref order and a gather
            uint32_t* segKeys = (uint32_t*)ctx->scratch[2].ptr;
            uint32_t* codesRef = (uint32_t*)ctx->scratch[3].ptr;
            k_morton<<<grid_for(N, kBlock), kBlock, 0, ctx->stream>>>(centroids, N, dBounds, codesRef, nullptr);
            k_segment_keys<<<grid_for(N, kBlock), kBlock, 0, ctx->stream>>>(centroids, order, N, segKeys);
            int bits = 1;
            while ((1 << bits) < nseg) bits++;
            // the sort needs its own two scratch arrays: reuse the node buffer (>= N-1 ints) is not enough, so allocate
            uint32_t* altK = nullptr;
            int32_t* altV = nullptr;
            if (!palloc(ctx, &altK, (size_t)N * 4) || !palloc(ctx, &altV, (size_t)N * 4)) {
                cudaGetLastError();
                pool_free(ctx, altK);
                return fail(set_error(MC_ERR_OOM, "mc_bvh_build_batch: sort scratch allocation failed"));
            }
            st = radix_sort_pairs(ctx, segKeys, order, altK, altV, N, bits);
            pool_free(ctx, altK);
            pool_free(ctx, altV);
            if (st != MC_OK) return fail(st);
            k_gather_u32<<<grid_for(N, kBlock), kBlock, 0, ctx->stream>>>(codesRef, order, N, bvh->codes, ctx->d_error);
        }
    }
    {
        // the hierarchy is only built over a valid sorted order
        int pre = 0;
        if ((st = flags_now(ctx, &pre)) != MC_OK) return fail(st);
        if (pre & MC_DEVERR_INPUT)
            return fail(set_error(MC_ERR_INVALID, "mc_bvh_build: the permutation is not a sorting permutation of the primitives"));
        if (pre) return fail(status_from_device_flags(pre));
    }
    if (cudaMemsetAsync(counters, 0, (size_t)nodesCount * 4, ctx->stream) != cudaSuccess ||
        cudaMemsetAsync(bvh->parents, 0xFF, (size_t)(NI + N) * 4, ctx->stream) != cudaSuccess)
        return fail(cuda_error(cudaGetLastError(), "memset", __FILE__, __LINE__));
    if (NI > 0)
        k_karras<<<grid_for(NI, kBlock), kBlock, 0, ctx->stream>>>(bvh->codes, dSeg, nseg, NI, (float4*)bvh->nodes,
                                                                  bvh->parents, bvh->ref_internal, bvh->ref_leaves,
                                                                  (int2*)ctx->scratch[1].ptr);
    k_leaves_refit<<<grid_for(N, kBlock), kBlock, 0, ctx->stream>>>(order, boundsRef, N, NI, dSeg, nseg, (float4*)bvh->nodes,
                                                                   (float4*)bvh->prims, bvh->parents, counters, bvh->ids,
                                                                   bvh->types, bvh->ref_internal, bvh->ref_leaves,
                                                                   dRootBoxes, ctx->d_error);
    if (N == 1) k_single_root<<<1, 1, 0, ctx->stream>>>((float4*)bvh->nodes, boundsRef);
    if (cudaGetLastError() != cudaSuccess) return fail(set_error(MC_ERR_CUDA, "mc_bvh_build: launch failed"));
    int flags = 0;
    bvh->seg_bounds.resize(nseg);
    if (cudaMemcpyAsync(bvh->seg_bounds.data(), dRootBoxes, (size_t)nseg * sizeof(mc_aabb), cudaMemcpyDeviceToHost,
                        ctx->stream) != cudaSuccess)
        return fail(cuda_error(cudaGetLastError(), "mc_bvh_build", __FILE__, __LINE__));
    if ((st = flags_now(ctx, &flags)) != MC_OK) return fail(st);
    if (flags) return fail(status_from_device_flags(flags));
    bvh->bounds = bvh->seg_bounds[0];
    bvh->seg_prim_off.resize(nseg);
    bvh->bin_roots.resize(nseg);
    for (int s = 0; s < nseg; s++) {
        bvh->seg_prim_off[s] = segs[s].primOff;
        bvh->bin_roots[s] = segs[s].intOff;
    }
    if (o.layout == MC_BVH_LAYOUT_WIDE4 || o.layout == MC_BVH_LAYOUT_WIDE4Q) {
        const bool coop = o.phase_launches == 0;
        // the wide layouts traverse the collapse of the clustered tree, or of
        // the LBVH when clustering does not apply (a one-primitive scene, a
        // collapse too deep for the stack) or the caller asks for it
        st = MC_ERR_UNSUPPORTED;
        if (o.builder == MC_BVH_BUILDER_CLUSTERED) {
            ClusterTree tree;
            st = build_ploc(ctx, bvh, dSeg, nseg, order, boundsRef, tree, coop);
            if (st == MC_OK) {
                st = build_wide(ctx, bvh, dSeg, nseg, dWideRoot, coop, tree.nodes, &tree.roots);
                pool_free(ctx, tree.nodes);
                if (st == MC_OK) bvh->builder = MC_BVH_BUILDER_CLUSTERED;
            }
            if (st != MC_OK && st != MC_ERR_UNSUPPORTED) return fail(st);
        }
        if (st == MC_ERR_UNSUPPORTED) {
            if (bvh->wide_nodes) pool_free(ctx, bvh->wide_nodes);
            if (bvh->wide_prims) pool_free(ctx, bvh->wide_prims);
            bvh->wide_nodes = bvh->wide_prims = nullptr;
            if ((st = build_wide(ctx, bvh, dSeg, nseg, dWideRoot, coop)) != MC_OK) return fail(st);
            bvh->builder = MC_BVH_BUILDER_LBVH;
        }
    }
    if (o.layout == MC_BVH_LAYOUT_WIDE4Q) {
        void* q = nullptr;
        if (!palloc(ctx, &q, (size_t)bvh->wide_count * 64)) {
            cudaGetLastError();
            return fail(set_error(MC_ERR_OOM, "mc_bvh_build: quantised-node allocation failed"));
        }
        k_quantize_wide<<<grid_for((int)bvh->wide_count, kBlock), kBlock, 0, ctx->stream>>>(
            (const float4*)bvh->wide_nodes, (int)bvh->wide_count, (float4*)q);
        if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
            pool_free(ctx, q);
            return fail(cuda_error(cudaGetLastError(), "mc_bvh_build (quantise)", __FILE__, __LINE__));
        }
        pool_free(ctx, bvh->wide_nodes);
        bvh->wide_nodes = q;
        bvh->layout = MC_BVH_LAYOUT_WIDE4Q;
    }
    *out = bvh;
    return MC_OK;
}

}  // namespace mc

extern "C" {

mc_status mc_morton_codes(mc_context* ctx, const mc_scene_view* scene, uint32_t* d_codes, mc_aabb* bounds_out) {
    if (!ctx || !d_codes) return mc::set_error(MC_ERR_INVALID, "mc_morton_codes: null argument");
    mc_status st = mc::check_scene(scene);
    if (st != MC_OK) return st;
    int n = scene->sphere_count + scene->triangle_count;
    if ((st = mc::devbuf_reserve(ctx->scratch[0], (size_t)n * sizeof(mc_aabb))) != MC_OK) return st;
    if ((st = mc::devbuf_reserve(ctx->scratch[1], (size_t)n * sizeof(float4))) != MC_OK) return st;
    std::vector<Seg> segs;
    Seg* dSeg;
    int* dBounds;
    mc_aabb* dRootBoxes;
    int* dWideRoot;
    if ((st = mc::upload_segments(ctx, scene, 1, segs, &dSeg, &dBounds, &dRootBoxes, &dWideRoot)) != MC_OK) return st;
    k_prim_bounds<<<grid_for(n, kBlock), kBlock, 0, ctx->stream>>>(dSeg, 1, n, (mc_aabb*)ctx->scratch[0].ptr,
                                                                  (float4*)ctx->scratch[1].ptr, dBounds);
    k_morton<<<grid_for(n, kBlock), kBlock, 0, ctx->stream>>>((const float4*)ctx->scratch[1].ptr, n, dBounds, d_codes, nullptr);
    MC_CUDA(cudaGetLastError());
    int h[6];
    MC_CUDA(cudaMemcpyAsync(h, dBounds, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    MC_CUDA(cudaStreamSynchronize(ctx->stream));
    if (bounds_out) {
        bounds_out->lo = mc_vec3{ordered_to_float(h[0]), ordered_to_float(h[1]), ordered_to_float(h[2])};
        bounds_out->hi = mc_vec3{ordered_to_float(h[3]), ordered_to_float(h[4]), ordered_to_float(h[5])};
        bounds_out->pad0 = bounds_out->pad1 = 0.f;
    }
    return MC_OK;
}

mc_status mc_radix_sort_pairs(mc_context* ctx, uint32_t* d_keys, int32_t* d_values, int32_t n, int32_t key_bits) {
    if (!ctx || (n > 0 && (!d_keys || !d_values)) || n < 0) return mc::set_error(MC_ERR_INVALID, "mc_radix_sort_pairs: bad argument");
    if (n >= (1 << 30)) return mc::set_error(MC_ERR_INVALID, "mc_radix_sort_pairs: n must be < 2^30");
    if (key_bits < 1 || key_bits > 32) return mc::set_error(MC_ERR_INVALID, "mc_radix_sort_pairs: key_bits must be in [1, 32]");
    mc_status st;
    if ((st = mc::devbuf_reserve(ctx->scratch[2], (size_t)n * 4 + 16)) != MC_OK) return st;
    if ((st = mc::devbuf_reserve(ctx->scratch[3], (size_t)n * 4 + 16)) != MC_OK) return st;
    MC_CUDA(cudaMemsetAsync(ctx->d_error, 0, sizeof(int), ctx->stream));
    st = mc::radix_sort_pairs(ctx, d_keys, d_values, (uint32_t*)ctx->scratch[2].ptr, (int32_t*)ctx->scratch[3].ptr, n, key_bits);
    if (st != MC_OK) return st;
    int flags = 0;
    if ((st = mc::flags_now(ctx, &flags)) != MC_OK) return st;
    return mc::status_from_device_flags(flags);
}

mc_status mc_radix_sort_pairs_static(mc_context* ctx, uint32_t* d_keys, int32_t* d_values, int32_t n, int32_t key_bits) {
    if (!ctx || (n > 0 && (!d_keys || !d_values)) || n < 0) return mc::set_error(MC_ERR_INVALID, "mc_radix_sort_pairs_static: bad argument");
    if (key_bits < 1 || key_bits > 32) return mc::set_error(MC_ERR_INVALID, "mc_radix_sort_pairs_static: key_bits must be in [1, 32]");
    if (n > MC_SORT_STATIC_MAX_PAIRS)
        return mc::set_error(MC_ERR_INVALID, "mc_radix_sort_pairs_static: n = %d exceeds the fixed scratch of %d pairs (use mc_radix_sort_pairs)",
                             n, MC_SORT_STATIC_MAX_PAIRS);
    if (n > 1) MC_CUDA(cudaMemsetAsync(ctx->d_error, 0, sizeof(int), ctx->stream));
    mc_status st = mc::radix_sort_pairs_static(ctx, d_keys, d_values, n, key_bits);
    if (st != MC_OK || n <= 1) return st;
    int flags = 0;
    if ((st = mc::flags_now(ctx, &flags)) != MC_OK) return st;
    return mc::status_from_device_flags(flags);
}

mc_status mc_bvh_build(mc_context* ctx, const mc_scene_view* scene, const mc_bvh_build_opts* opts, mc_bvh** out) {
    if (!scene) return mc::set_error(MC_ERR_INVALID, "mc_bvh_build: null scene");
    return mc::build_segments(ctx, scene, 1, opts, out);
}

mc_status mc_bvh_build_batch(mc_context* ctx, const mc_scene_view* scenes, int32_t count, const mc_bvh_build_opts* opts,
                             mc_bvh** out) {
    if (!scenes || count < 1) return mc::set_error(MC_ERR_INVALID, "mc_bvh_build_batch: no scenes");
    return mc::build_segments(ctx, scenes, count, opts, out);
}

mc_status mc_bvh_free(mc_bvh* bvh) {
    if (!bvh) return MC_OK;
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != bvh->device) cudaSetDevice(bvh->device);
    // work on any stream may still read the tree (cudaFree would wait for the device too)
    cudaDeviceSynchronize();
    void* bufs[] = {bvh->nodes, bvh->prims, bvh->wide_nodes, bvh->wide_prims, bvh->codes,
                    bvh->ids, bvh->types, bvh->parents, bvh->ref_internal, bvh->ref_leaves};
    for (void* b : bufs) mc::pool_release(b);
    if (prev >= 0 && prev != bvh->device) cudaSetDevice(prev);
    delete bvh;
    return MC_OK;
}

mc_status mc_bvh_get_info(const mc_bvh* bvh, mc_bvh_info* info) {
    if (!bvh || !info) return mc::set_error(MC_ERR_INVALID, "mc_bvh_get_info: null argument");
    mc_status st = mc::bvh_depth(const_cast<mc_bvh*>(bvh));
    if (st != MC_OK) return st;
    info->primitive_count = bvh->n;
    info->internal_count = bvh->ni;
    info->depth = bvh->depth;
    info->layout = bvh->layout;
    info->node_bytes = bvh->layout == MC_BVH_LAYOUT_WIDE4    ? bvh->wide_count * 128
                       : bvh->layout == MC_BVH_LAYOUT_WIDE4Q ? bvh->wide_count * 64
                                                             : bvh->node_bytes;
    info->prim_bytes = (long long)bvh->n * 48;
    info->scene_bounds = bvh->bounds;
    info->wide_levels = bvh->layout != MC_BVH_LAYOUT_BINARY && bvh->wide_levels > 0 ? bvh->wide_levels : 0;
    return MC_OK;
}

mc_status mc_bvh_export(const mc_bvh* bvh, uint32_t* d_codes, int32_t* d_ids, int32_t* d_types, mc_bvh_node* d_internal,
                        mc_bvh_node* d_leaves) {
    if (!bvh) return mc::set_error(MC_ERR_INVALID, "mc_bvh_export: null bvh");
    cudaStream_t s = bvh->ctx->stream;
    int n = bvh->n;
    if (d_codes) MC_CUDA(cudaMemcpyAsync(d_codes, bvh->codes, (size_t)n * 4, cudaMemcpyDeviceToDevice, s));
    if (d_ids) MC_CUDA(cudaMemcpyAsync(d_ids, bvh->ids, (size_t)n * 4, cudaMemcpyDeviceToDevice, s));
    if (d_types) MC_CUDA(cudaMemcpyAsync(d_types, bvh->types, (size_t)n * 4, cudaMemcpyDeviceToDevice, s));
    if (d_internal || d_leaves) {
        if (!bvh->ref_internal) return mc::set_error(MC_ERR_INVALID, "mc_bvh_export: build with keep_reference_nodes to export nodes");
        if (d_internal && n > 1)
            MC_CUDA(cudaMemcpyAsync(d_internal, bvh->ref_internal, (size_t)(n - 1) * sizeof(mc_bvh_node), cudaMemcpyDeviceToDevice, s));
        if (d_leaves) MC_CUDA(cudaMemcpyAsync(d_leaves, bvh->ref_leaves, (size_t)n * sizeof(mc_bvh_node), cudaMemcpyDeviceToDevice, s));
    }
    MC_CUDA(cudaStreamSynchronize(s));
    return MC_OK;
}

mc_status mc_bvh_export_traversal(const mc_bvh* bvh, void* d_nodes, void* d_prims) {
    if (!bvh) return mc::set_error(MC_ERR_INVALID, "mc_bvh_export_traversal: null bvh");
    cudaStream_t s = bvh->ctx->stream;
    const bool wide = bvh->layout != MC_BVH_LAYOUT_BINARY;
    const long long nodeBytes = bvh->layout == MC_BVH_LAYOUT_WIDE4    ? bvh->wide_count * 128
                                : bvh->layout == MC_BVH_LAYOUT_WIDE4Q ? bvh->wide_count * 64
                                                                      : bvh->node_bytes;
    if (d_nodes && nodeBytes > 0)
        MC_CUDA(cudaMemcpyAsync(d_nodes, wide ? bvh->wide_nodes : bvh->nodes, (size_t)nodeBytes, cudaMemcpyDeviceToDevice, s));
    if (d_prims && bvh->n > 0)
        MC_CUDA(cudaMemcpyAsync(d_prims, wide ? bvh->wide_prims : bvh->prims, (size_t)bvh->n * 48, cudaMemcpyDeviceToDevice, s));
    MC_CUDA(cudaStreamSynchronize(s));
    return MC_OK;
}

}  // extern "C"
