// mc_guide.cu - the path-guiding MLP on the sm_100a tensor cores.
//
// Network: 144 encoded inputs -> 64 -> 64 -> 64 (ReLU) -> 40 outputs (an
// 8-lobe vMF mixture). Every layer is a tcgen05.mma (kind::f16, BF16 operands
// from shared memory, FP32 accumulators in tensor memory) over a tile of 128
// queries, issued by one thread; the 128 threads of the CTA each own one
// query row for the epilogues (TMEM -> registers -> ReLU -> BF16 -> shared
// memory as the next layer's operand). Each bias is folded into its layer's
// MMA (a [1, 1, 0...] column block on the activations against a
// [hi, lo, 0...] block on the weights), so a forward epilogue is one
// ReLU-and-convert instruction per pair of columns.
//
// Training (one kernel, forward + backward per tile of 128 records):
//   forward   Z_l = [H_{l-1} | 1 1 0..] Wb_l^T   (A = activations, B = Wb_l)
//   loss      -w log q(next) of the vMF mixture, gradient dY per row (FP32)
//   backward  dH_{l-1} = dZ_l W_l                (A = dZ_l, B = Wb_l read
//                                                 MN-major)
//             dW_l += dZ_l^T [H_{l-1} | 1 1 0..] (A = the dZ_l rows read
//                                                 MN-major as 128 output
//                                                 rows, the upper ones zero;
//                                                 B = the activation rows read
//                                                 MN-major; the first ones
//                                                 column gives the bias
//                                                 gradient)
// Reading the stored rows MN-major replaces every transposed copy. The weight
// gradients accumulate in tensor memory over all tiles a CTA processes (464
// of the 512 columns) and are written once per CTA as FP32 partials; the Adam
// kernel sums the partials in a fixed order (deterministic) and updates FP32
// master weights, from which the BF16 operands are regenerated.
//
// Compiled without fast math: the encoding and the loss are compared with an
// FP64 restatement.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "mc_guide.cuh"
#include "mc_internal.h"
#include "mc_umma.cuh"

#define MC_CUDA(call)                                                                      \
    do {                                                                                   \
        cudaError_t e__ = (call);                                                          \
        if (e__ != cudaSuccess) return mc::cuda_error((int)e__, #call, __FILE__, __LINE__); \
    } while (0)

namespace {

using namespace mc::guide;
using namespace mc::umma;
typedef __nv_bfloat16 bf16;

constexpr int kTile = 128;
constexpr long long kWaitLimit = 1ll << 20;

// ---- shared-memory layouts (bytes) ----
// inference (bias-folded operands: inputs of kInK and kHidK columns)
constexpr int iW1 = 0;
constexpr int iW2 = iW1 + kHid * kInK * 2;
constexpr int iW3 = iW2 + kHid * kHidK * 2;
constexpr int iW4 = iW3 + kHid * kHidK * 2;
// kInferGroups warpgroups per CTA share one copy of the weights; each has its
// own tile buffer (the encoded inputs X0, then in place each hidden layer's
// activations once the MMA that read the previous contents has finished) and
// its own 64 TMEM columns, so while one group waits on its MMA the others run
// their epilogues.
constexpr int kInferGroups = 4;
constexpr int iTiles = iW4 + kOutPad * kHidK * 2;
constexpr int kInferTileBytes = kTile * kInK * 2;
constexpr int kInferSmem = iTiles + kInferGroups * kInferTileBytes;
static_assert(iTiles % 128 == 0 && kInferTileBytes % 128 == 0, "operand buffers must stay aligned");
static_assert(kTile * kHidK * 2 <= kInferTileBytes, "the activations fit the input buffer");
static_assert(kInferSmem <= 232448 - 1024, "inference CTA exceeds the shared memory of one CTA");
// training: the inference operands (bias-folded weights, encoded inputs and
// activations with their bias blocks), plus the gradient rows
constexpr int tW1 = 0;
constexpr int tW2 = tW1 + kHid * kInK * 2;
constexpr int tW3 = tW2 + kHid * kHidK * 2;
constexpr int tW4 = tW3 + kHid * kHidK * 2;
constexpr int kDCols = 128;                             // gradient rows: dY or dZ in 0..63, zeros above
constexpr int tD = tW4 + kOutPad * kHidK * 2;
constexpr int tX = tD + kTile * kDCols * 2;             // encoded inputs + bias block (128 x 160)
constexpr int tH1 = tX + kTile * kInK * 2;              // activations + bias block (128 x 80)
constexpr int tH2 = tH1 + kTile * kHidK * 2;
constexpr int tH3 = tH2 + kTile * kHidK * 2;
// The MN-major reads span the whole of each buffer; a buffer is followed by
// at least 9 KB more of the allocation (the tail after tH3), which an MN-major
// read with its two descriptor strides exchanged would also stay inside.
constexpr int kTrainSmem = tH3 + kTile * kHidK * 2 + 9216;
static_assert(tD % 128 == 0 && tX % 128 == 0 && tH1 % 128 == 0, "operand buffers must stay aligned");
static_assert(kTrainSmem <= 232448 - 1024, "training tile exceeds the shared memory of one CTA");

// TMEM columns of the training kernel
constexpr uint32_t cR = 0, cG1 = 64, cG2 = 224, cG3 = 304, cG4 = 384, kTrainCols = 512;
constexpr uint32_t kInferCols = 64 * kInferGroups;

struct GuideInferArgs {
    const bf16* blob;
    const float* master;
    float lox, loy, loz, invx, invy, invz;
    int n;
    const int* count;
    int capacity;
    const float* queries;                   // API: n x 6
    const int* queue;                       // render: path per slot
    const float *ox, *oy, *oz, *dx, *dy, *dz, *time;
    const mc_packed_hit* hits;
    const mc_triangle_hot* hot;             // render with MC_GUIDE_DIR_NORMAL: the hit primitives
    const mc_sphere* spheres;
    int dirNormal;
    int stride;                             // > 1: one query per `stride` queue slots (the first of each run)
    float anchor;                           // anchored lobes: this times the direction input offsets every raw mean
    float* mix;
    int* err;
};

// Geometric normal of the hit primitive, turned to face the arriving ray d
// (the shade kernel's face normal: e1 x e2 for a triangle, centre to hit point
// for a sphere at the ray's time).
__device__ __forceinline__ void face_normal(const GuideInferArgs& a, int type, int idx, float t, float time, float px,
                                            float py, float pz, float dx, float dy, float dz, float* n) {
    float nx, ny, nz;
    if (type == 1) {
        const float* v = reinterpret_cast<const float*>(a.hot + idx);
        const float e1x = v[3] - v[0], e1y = v[4] - v[1], e1z = v[5] - v[2];
        const float e2x = v[6] - v[0], e2y = v[7] - v[1], e2z = v[8] - v[2];
        nx = e1y * e2z - e1z * e2y;
        ny = e1z * e2x - e1x * e2z;
        nz = e1x * e2y - e1y * e2x;
    } else {
        const mc_sphere& sp = a.spheres[idx];
        float cx = sp.center.x, cy = sp.center.y, cz = sp.center.z;
        if (sp.is_moving) {
            cx = cx + (sp.center1.x - cx) * time;
            cy = cy + (sp.center1.y - cy) * time;
            cz = cz + (sp.center1.z - cz) * time;
        }
        nx = px - cx; ny = py - cy; nz = pz - cz;
    }
    const float len = sqrtf(nx * nx + ny * ny + nz * nz);
    if (!(len > 0.f)) {
        n[0] = -dx; n[1] = -dy; n[2] = -dz;
        return;
    }
    const float r = 1.0f / len;
    nx = nx * r; ny = ny * r; nz = nz * r;
    if (dx * nx + dy * ny + dz * nz >= 0.f) {
        nx = -nx; ny = -ny; nz = -nz;
    }
    n[0] = nx; n[1] = ny; n[2] = nz;
}

struct GuideTrainArgs {
    const bf16* blob;
    const float* master;
    float lox, loy, loz, invx, invy, invz;
    const float* records;                   // already advanced to this step's slice
    int n;
    const int* count;                       // device count of the whole batch (or null: n records)
    int offset;                             // this step's first record in the batch
    int capacity;                           // records the batch holds
    int stepCap;                            // records one step takes
    const float* scale;
    float weightCap;                        // > 0: a record's normalized weight is at most weightCap / n
    float anchor;                           // anchored lobes (GuideInferArgs::anchor)
    float* partials;
    double* loss;
    int* err;
};

__device__ __forceinline__ void sync_operands() {
    fence_async_smem();
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
}

// Thread 0 waits for the committed MMAs; every thread learns the outcome.
__device__ __forceinline__ bool wait_mma(uint64_t* bar, uint32_t& phase, int* sFlag, int* err) {
    if (threadIdx.x == 0) {
        bool ok = mbar_wait(bar, phase, kWaitLimit);
        *sFlag = ok ? 0 : 1;
        if (!ok) atomicOr(err, MC_DEVERR_TIMEOUT);
    }
    __syncthreads();
    fence_after_sync();
    if (*sFlag) return false;
    phase ^= 1u;
    return true;
}

__device__ __forceinline__ void load_kmaj(unsigned char* dst, const bf16* src, int rows, int K) {
    const int per = K / 8;
    for (int c = threadIdx.x; c < rows * per; c += blockDim.x) {
        int r = c / per, k8 = (c % per) * 8;
        *reinterpret_cast<uint4*>(dst + kmaj_off(r, k8, K)) = *reinterpret_cast<const uint4*>(src + (size_t)r * K + k8);
    }
}

// TMEM address of column c of this warp's 32-lane slice (warp w of a
// warpgroup reads lanes 32 (w % 4) .. 32 (w % 4) + 31).
__device__ __forceinline__ uint32_t tcol(uint32_t base, uint32_t c) {
    return base + ((uint32_t)(threadIdx.x & 96) << 16) + c;
}

// Barrier of the 128 threads of warpgroup g (named barrier 1 + g).
__device__ __forceinline__ void wg_sync(int g) { asm volatile("bar.sync %0, 128;" ::"r"(1 + g) : "memory"); }

__device__ __forceinline__ void wg_sync_operands(int g) {
    fence_async_smem();
    fence_before_sync();
    wg_sync(g);
    fence_after_sync();
}

// The group's first thread waits for its committed MMAs; the group learns the outcome.
__device__ __forceinline__ bool wg_wait_mma(int g, uint64_t* bar, uint32_t& phase, int* sFlag, int* err) {
    if ((threadIdx.x & 127) == 0) {
        bool ok = mbar_wait(bar, phase, kWaitLimit);
        *sFlag = ok ? 0 : 1;
        if (!ok) atomicOr(err, MC_DEVERR_TIMEOUT);
    }
    wg_sync(g);
    fence_after_sync();
    if (*sFlag) return false;
    phase ^= 1u;
    return true;
}

// The bias block [1, 1, 0, ...] of a bias-folded operand row (columns k0..k0+15).
__device__ __forceinline__ void store_bias_block(unsigned char* s, int row, int k0, int K) {
    *reinterpret_cast<uint4*>(s + kmaj_off(row, k0, K)) = make_uint4(0x3F803F80u, 0u, 0u, 0u);  // bf16 1.0 twice
    *reinterpret_cast<uint4*>(s + kmaj_off(row, k0 + 8, K)) = make_uint4(0u, 0u, 0u, 0u);
}

// Encodes one query row into a K-major X0 operand of K columns (kIn, or kInK
// with the bias block after the inputs).
__device__ __forceinline__ void encode_row(unsigned char* sE, int row, const float* coord6, int K) {
#pragma unroll
    for (int c = 0; c < 6; c++) {
        float f[24];
        encode_coord(coord6[c], f);
#pragma unroll
        for (int j = 0; j < 3; j++)
            *reinterpret_cast<uint4*>(sE + kmaj_off(row, 24 * c + 8 * j, K)) = pack8_bf16(f + 8 * j);
    }
    if (K == kInK) store_bias_block(sE, row, kIn, K);
}

// Hidden-layer epilogue of the bias-folded network: 64 accumulator columns
// (bias included), ReLU and BF16 in one conversion, written as the next
// layer's operand row with its bias block.
__device__ __forceinline__ void epi_relu(uint32_t tR, unsigned char* sOut, int row) {
#pragma unroll
    for (int c = 0; c < kHid; c += 32) {
        uint32_t v[32];
        tmem_ld32(tcol(tR, c), v);
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const uint32_t* w = v + 8 * q;
            uint4 u;
            u.x = relu_bf16x2(__uint_as_float(w[0]), __uint_as_float(w[1]));
            u.y = relu_bf16x2(__uint_as_float(w[2]), __uint_as_float(w[3]));
            u.z = relu_bf16x2(__uint_as_float(w[4]), __uint_as_float(w[5]));
            u.w = relu_bf16x2(__uint_as_float(w[6]), __uint_as_float(w[7]));
            *reinterpret_cast<uint4*>(sOut + kmaj_off(row, c + 8 * q, kHidK)) = u;
        }
    }
    store_bias_block(sOut, row, kHid, kHidK);
}

// Raw outputs -> mixture (weights, unit means, kappa). anc: the anchor
// offset added to every raw mean (zero for unanchored guides).
__device__ __forceinline__ void raw_to_mixture(const float* y, const float* anc, float* m) {
    float mx = y[0];
#pragma unroll
    for (int k = 1; k < kLobes; k++) mx = fmaxf(mx, y[k]);
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < kLobes; k++) {
        m[k] = expf(y[k] - mx);
        s += m[k];
    }
    const float invS = 1.0f / s;
#pragma unroll
    for (int k = 0; k < kLobes; k++) {
        m[k] = m[k] * invS;
        float a = y[8 + 3 * k] + anc[0], b = y[9 + 3 * k] + anc[1], c = y[10 + 3 * k] + anc[2];
        float len = sqrtf(a * a + b * b + c * c);
        if (len > 1e-20f) {
            const float r = 1.0f / len;
            m[8 + 3 * k] = a * r; m[9 + 3 * k] = b * r; m[10 + 3 * k] = c * r;
        } else {
            m[8 + 3 * k] = 0.f; m[9 + 3 * k] = 0.f; m[10 + 3 * k] = 1.f;
        }
        m[32 + k] = expf(fminf(fmaxf(y[32 + k], kLogKappaMin), kLogKappaMax));
    }
}

// Loss -W log q(w) of one record and its gradient w.r.t. the 40 raw outputs
// (the anchor offset anc is a constant: a raw mean's gradient is its
// anchored mean's).
__device__ float loss_grad(const float* y, const float* anc, float wx, float wy, float wz, float W, float* dy) {
    float mx = y[0];
    for (int k = 1; k < kLobes; k++) mx = fmaxf(mx, y[k]);
    float e[kLobes], s = 0.f;
    for (int k = 0; k < kLobes; k++) {
        e[k] = expf(y[k] - mx);
        s += e[k];
    }
    float wk[kLobes], vk[kLobes], kap[kLobes], cs[kLobes], len[kLobes], mu[3 * kLobes];
    bool clamped[kLobes];
    float q = 0.f;
    for (int k = 0; k < kLobes; k++) {
        wk[k] = e[k] / s;
        float a = y[8 + 3 * k] + anc[0], b = y[9 + 3 * k] + anc[1], c = y[10 + 3 * k] + anc[2];
        float l = sqrtf(a * a + b * b + c * c);
        if (l > 1e-20f) {
            mu[3 * k] = a / l; mu[3 * k + 1] = b / l; mu[3 * k + 2] = c / l;
        } else {
            mu[3 * k] = 0.f; mu[3 * k + 1] = 0.f; mu[3 * k + 2] = 1.f;
            l = 0.f;
        }
        len[k] = l;
        float lk = y[32 + k];
        clamped[k] = lk < kLogKappaMin || lk > kLogKappaMax;
        kap[k] = expf(fminf(fmaxf(lk, kLogKappaMin), kLogKappaMax));
        cs[k] = mu[3 * k] * wx + mu[3 * k + 1] * wy + mu[3 * k + 2] * wz;
        vk[k] = vmf_pdf(kap[k], cs[k]);
        q += wk[k] * vk[k];
    }
    q = fmaxf(q, 1e-30f);
    for (int k = 0; k < kLobes; k++) {
        float r = wk[k] * vk[k] / q;
        dy[k] = -W * (r - wk[k]);
        float dlogv = 1.0f / kap[k] - 2.0f / expm1f(2.0f * kap[k]) + cs[k] - 1.0f;
        dy[32 + k] = clamped[k] ? 0.f : -W * r * kap[k] * dlogv;
        float g = len[k] > 0.f ? -W * r * kap[k] / len[k] : 0.f;
        dy[8 + 3 * k] = g * (wx - cs[k] * mu[3 * k]);
        dy[9 + 3 * k] = g * (wy - cs[k] * mu[3 * k + 1]);
        dy[10 + 3 * k] = g * (wz - cs[k] * mu[3 * k + 2]);
    }
    return W != 0.f ? -W * logf(q) : 0.f;
}

// ---------------------------------------------------------------------------
// Inference
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128 * kInferGroups, 1) k_guide_infer(GuideInferArgs a) {
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ uint64_t bars[kInferGroups];
    __shared__ uint32_t tbase;
    __shared__ int sFlags[kInferGroups];
    const int tid = threadIdx.x, g = tid >> 7, row = tid & 127;
    if ((tid >> 5) == 0) tmem_alloc(&tbase, kInferCols);
    if (tid < kInferGroups) {
        mbar_init(&bars[tid], 1);
        sFlags[tid] = 0;
    }
    load_kmaj(sm + iW1, a.blob + bI1, kHid, kInK);
    load_kmaj(sm + iW2, a.blob + bI2, kHid, kHidK);
    load_kmaj(sm + iW3, a.blob + bI3, kHid, kHidK);
    load_kmaj(sm + iW4, a.blob + bI4, kOutPad, kHidK);
    sync_operands();
    const uint32_t R = tbase + 64u * (uint32_t)g;
    const uint32_t s0 = smem_u32(sm);
    const uint32_t sX = s0 + iTiles + (uint32_t)g * kInferTileBytes;
    unsigned char* bufX = sm + iTiles + g * kInferTileBytes;
    uint64_t* bar = &bars[g];
    int* sFlag = &sFlags[g];
    const uint32_t id64 = idesc_bf16(128, kHid), id48 = idesc_bf16(128, kOutPad);
    const int nSlots = a.count ? min(*a.count, a.capacity) : a.n;
    const int n = a.stride > 1 ? (nSlots + a.stride - 1) / a.stride : nSlots;
    uint32_t phase = 0;
    bool ok = true;
    // the groups take tiles in turn; from here on a group synchronises only itself
    for (int tile = blockIdx.x * kInferGroups + g; tile * kTile < n; tile += gridDim.x * kInferGroups) {
        const int q = tile * kTile + row;
        const bool valid = q < n;
        float coord[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        int out = -1;
        if (valid) {
            float px, py, pz, dx, dy, dz;
            if (a.queue) {
                const int p = a.queue[a.stride > 1 ? q * a.stride : q];
                const int4 h = reinterpret_cast<const int4*>(a.hits)[p];
                const float t = h.w ? __int_as_float(h.x) : 0.f;
                dx = a.dx[p]; dy = a.dy[p]; dz = a.dz[p];
                px = a.ox[p] + dx * t; py = a.oy[p] + dy * t; pz = a.oz[p] + dz * t;
                if (a.dirNormal && h.w) {
                    float nrm[3];
                    face_normal(a, h.y, h.z, t, a.time[p], px, py, pz, dx, dy, dz, nrm);
                    dx = nrm[0]; dy = nrm[1]; dz = nrm[2];
                }
                out = p;
            } else {
                const float* Q = a.queries + (size_t)q * 6;
                px = Q[0]; py = Q[1]; pz = Q[2]; dx = Q[3]; dy = Q[4]; dz = Q[5];
                out = q;
            }
            coord[0] = (px - a.lox) * a.invx;
            coord[1] = (py - a.loy) * a.invy;
            coord[2] = (pz - a.loz) * a.invz;
            coord[3] = dx; coord[4] = dy; coord[5] = dz;
        }
        encode_row(bufX, row, coord, kInK);
        wg_sync_operands(g);
        if (row == 0) {
            gemm_k(R, sX, s0 + iW1, kInK, id64, 0);
            commit(bar);
        }
        if (!(ok = wg_wait_mma(g, bar, phase, sFlag, a.err))) break;
        epi_relu(R, bufX, row);  // the MMA that read X0 is done: H1 goes in its place
        wg_sync_operands(g);
        if (row == 0) {
            gemm_k(R, sX, s0 + iW2, kHidK, id64, 0);
            commit(bar);
        }
        if (!(ok = wg_wait_mma(g, bar, phase, sFlag, a.err))) break;
        epi_relu(R, bufX, row);
        wg_sync_operands(g);
        if (row == 0) {
            gemm_k(R, sX, s0 + iW3, kHidK, id64, 0);
            commit(bar);
        }
        if (!(ok = wg_wait_mma(g, bar, phase, sFlag, a.err))) break;
        epi_relu(R, bufX, row);
        wg_sync_operands(g);
        if (row == 0) {
            gemm_k(R, sX, s0 + iW4, kHidK, id48, 0);
            commit(bar);
        }
        if (!(ok = wg_wait_mma(g, bar, phase, sFlag, a.err))) break;
        float y[kOutPad];
        {
            uint32_t v[32];
            tmem_ld32(tcol(R, 0), v);
#pragma unroll
            for (int k = 0; k < 32; k++) y[k] = __uint_as_float(v[k]);
        }
        tmem_ld16(tcol(R, 32), y + 32);
        if (valid) {
            float m[kOut];
            const float anc[3] = {a.anchor * coord[3], a.anchor * coord[4], a.anchor * coord[5]};
            raw_to_mixture(y, anc, m);
            float4* dst = reinterpret_cast<float4*>(a.mix + (size_t)out * kOut);
            for (int i = 0; i < kOut / 4; i++) dst[i] = make_float4(m[4 * i], m[4 * i + 1], m[4 * i + 2], m[4 * i + 3]);
        }
        // the next tile's operand barrier (fenced) orders these TMEM reads before its MMA
    }
    fence_before_sync();
    __syncthreads();
    if (!ok && row == 0) mbar_wait(bar, phase, kWaitLimit);  // let an overdue MMA finish before TMEM goes back
    __syncthreads();
    if ((tid >> 5) == 0) tmem_dealloc(tbase, kInferCols);
}

// ---------------------------------------------------------------------------
// Training: forward + loss + backward, weight gradients accumulated in TMEM
// ---------------------------------------------------------------------------
// dZ = dH * relu'(Z) for one row: 64 accumulator columns, kept where the
// stored activation is positive, BF16 into columns 0..63 of the gradient row.
__device__ __forceinline__ void relu_grad(uint32_t tR, const unsigned char* sH, unsigned char* sD, int row) {
#pragma unroll
    for (int c = 0; c < kHid; c += 32) {
        uint32_t v[32];
        tmem_ld32(tcol(tR, c), v);
#pragma unroll
        for (int q = 0; q < 4; q++) {
            float h[8], g[8];
            unpack8_bf16(*reinterpret_cast<const uint4*>(sH + kmaj_off(row, c + 8 * q, kHidK)), h);
#pragma unroll
            for (int j = 0; j < 8; j++) g[j] = h[j] > 0.f ? __uint_as_float(v[8 * q + j]) : 0.f;
            *reinterpret_cast<uint4*>(sD + kmaj_off(row, c + 8 * q, kDCols)) = pack8_bf16(g);
        }
    }
}

__global__ void __launch_bounds__(128, 1) k_guide_train(GuideTrainArgs a) {
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ uint64_t bar;
    __shared__ uint32_t tbase;
    __shared__ int sFlag;
    const int tid = threadIdx.x, warp = tid >> 5, row = tid;
    if (warp == 0) tmem_alloc(&tbase, kTrainCols);
    if (tid == 0) {
        mbar_init(&bar, 1);
        sFlag = 0;
    }
    // the bias-folded forward weights; read MN-major they are also the data
    // gradients' B operands (W instead of a transposed copy)
    load_kmaj(sm + tW1, a.blob + bI1, kHid, kInK);
    load_kmaj(sm + tW2, a.blob + bI2, kHid, kHidK);
    load_kmaj(sm + tW3, a.blob + bI3, kHid, kHidK);
    load_kmaj(sm + tW4, a.blob + bI4, kOutPad, kHidK);
    // columns 64..127 of the gradient rows stay zero: the weight-gradient MMAs
    // read them as output units 64..127 of an M = 128 tile
    for (int i = tid; i < kTile * 8; i += blockDim.x)
        *reinterpret_cast<uint4*>(sm + tD + kmaj_off(i >> 3, kHid + 8 * (i & 7), kDCols)) = make_uint4(0u, 0u, 0u, 0u);
    sync_operands();

    const uint32_t T = tbase;
    const uint32_t s0 = smem_u32(sm);
    const uint32_t id64 = idesc_bf16(128, kHid), id48 = idesc_bf16(128, kOutPad);
    // data gradients dH = dZ W: A = gradient rows (K-major over outputs), B = W read MN-major
    const uint32_t idData = id64 | kMajorB_MN;
    // weight gradients dW += dZ^T [H | 1 1 0..]: both operands read MN-major, K = the tile's records
    const uint32_t idW80 = idesc_bf16(128, kHidK) | kMajorA_MN | kMajorB_MN;
    const uint32_t idW160 = idesc_bf16(128, kInK) | kMajorA_MN | kMajorB_MN;
    const Operand gradRows = kmajor(s0 + tD, kDCols), gradCols = mnmajor(s0 + tD, kDCols);
    const int n = a.count ? max(0, min(min(*a.count, a.capacity) - a.offset, a.stepCap)) : a.n;
    const float scale = a.scale ? *a.scale : 1.0f;
    uint32_t phase = 0;
    bool ok = true;
    int done = 0;
    float lossAcc = 0.f;
    for (int tile = blockIdx.x; tile * kTile < n; tile += gridDim.x) {
        const int q = tile * kTile + row;
        const bool valid = q < n;
        float rec[MC_GUIDE_RECORD_FLOATS];
        for (int i = 0; i < MC_GUIDE_RECORD_FLOATS; i++) rec[i] = valid ? a.records[(size_t)q * MC_GUIDE_RECORD_FLOATS + i] : 0.f;
        float coord[6];
        coord[0] = (rec[0] - a.lox) * a.invx;
        coord[1] = (rec[1] - a.loy) * a.invy;
        coord[2] = (rec[2] - a.loz) * a.invz;
        coord[3] = rec[3]; coord[4] = rec[4]; coord[5] = rec[5];
        if (!valid) for (int i = 0; i < 6; i++) coord[i] = 0.f;
        encode_row(sm + tX, row, coord, kInK);
        sync_operands();
        // ---- forward (biases folded into the MMAs) ----
        if (tid == 0) {
            gemm_k(T + cR, s0 + tX, s0 + tW1, kInK, id64, 0);
            commit(&bar);
        }
        if (!(ok = wait_mma(&bar, phase, &sFlag, a.err))) break;
        epi_relu(T + cR, sm + tH1, row);
        sync_operands();
        if (tid == 0) {
            gemm_k(T + cR, s0 + tH1, s0 + tW2, kHidK, id64, 0);
            commit(&bar);
        }
        if (!(ok = wait_mma(&bar, phase, &sFlag, a.err))) break;
        epi_relu(T + cR, sm + tH2, row);
        sync_operands();
        if (tid == 0) {
            gemm_k(T + cR, s0 + tH2, s0 + tW3, kHidK, id64, 0);
            commit(&bar);
        }
        if (!(ok = wait_mma(&bar, phase, &sFlag, a.err))) break;
        epi_relu(T + cR, sm + tH3, row);
        sync_operands();
        if (tid == 0) {
            gemm_k(T + cR, s0 + tH3, s0 + tW4, kHidK, id48, 0);
            commit(&bar);
        }
        if (!(ok = wait_mma(&bar, phase, &sFlag, a.err))) break;
        // ---- loss and dY (columns kOut..63 zero) ----
        {
            float y[kOutPad];
            {
                uint32_t v[32];
                tmem_ld32(tcol(T + cR, 0), v);
#pragma unroll
                for (int k = 0; k < 32; k++) y[k] = __uint_as_float(v[k]);
            }
            tmem_ld16(tcol(T + cR, 32), y + 32);
            float dy[kHid];
            for (int k = kOut; k < kHid; k++) dy[k] = 0.f;
            float W = valid ? rec[9] * scale : 0.f;
            if (a.weightCap > 0.f && n > 0) W = fminf(W, a.weightCap / (float)n);
            const float anc[3] = {a.anchor * rec[3], a.anchor * rec[4], a.anchor * rec[5]};
            lossAcc += loss_grad(y, anc, rec[6], rec[7], rec[8], W, dy);
#pragma unroll
            for (int c = 0; c < kHid; c += 8)
                *reinterpret_cast<uint4*>(sm + tD + kmaj_off(row, c, kDCols)) = pack8_bf16(dy + c);
        }
        sync_operands();
        if (tid == 0) {
            gemm_op(T + cR, gradRows, mnmajor(s0 + tW4, kHidK), kOutPad, idData, 0);          // dH3 = dY W4
            gemm_op(T + cG4, gradCols, mnmajor(s0 + tH3, kHidK), kTile, idW80, done > 0);     // dW4 | db4
            commit(&bar);
        }
        if (!(ok = wait_mma(&bar, phase, &sFlag, a.err))) break;
        // ---- layers 3, 2: dZ = dH * relu'(Z), then the next data / weight gradients ----
        const int hOff[3] = {tH3, tH2, tH1};
        const int wOff[2] = {tW3, tW2};
        const uint32_t gOff[2] = {cG3, cG2};
        for (int l = 0; l < 2; l++) {
            relu_grad(T + cR, sm + hOff[l], sm + tD, row);
            sync_operands();
            if (tid == 0) {
                gemm_op(T + cR, gradRows, mnmajor(s0 + wOff[l], kHidK), kHid, idData, 0);
                gemm_op(T + gOff[l], gradCols, mnmajor(s0 + hOff[l + 1], kHidK), kTile, idW80, done > 0);
                commit(&bar);
            }
            if (!(ok = wait_mma(&bar, phase, &sFlag, a.err))) break;
        }
        if (!ok) break;
        // ---- layer 1: dZ1, then dW1 | db1 against the encoded inputs ----
        relu_grad(T + cR, sm + tH1, sm + tD, row);
        sync_operands();
        if (tid == 0) {
            gemm_op(T + cG1, gradCols, mnmajor(s0 + tX, kInK), kTile, idW160, done > 0);
            commit(&bar);
        }
        if (!(ok = wait_mma(&bar, phase, &sFlag, a.err))) break;
        done++;
    }
    // loss
    for (int off = 16; off > 0; off >>= 1) lossAcc += __shfl_xor_sync(0xffffffffu, lossAcc, off);
    if ((tid & 31) == 0 && a.loss && lossAcc != 0.f) atomicAdd(a.loss, (double)lossAcc);
    // per-CTA partial gradients (rows = output units, lanes 0..63)
    if (warp < 2) {
        const int o = row;
        float* P = a.partials + (size_t)blockIdx.x * kParams;
        const bool have = ok && done > 0;
        for (int c = 0; c < 160; c += 16) {
            float v[16];
            if (have) tmem_ld16(tcol(T + cG1, c), v);
            for (int j = 0; j < 16; j++) {
                const int i = c + j;
                const float g = have ? v[j] : 0.f;
                if (i < kIn) P[oW1 + o * kIn + i] = g;
                else if (i == kIn) P[oB1 + o] = g;
            }
        }
        const uint32_t gc[3] = {cG2, cG3, cG4};
        const int ow[3] = {oW2, oW3, oW4}, ob[3] = {oB2, oB3, oB4};
        for (int l = 0; l < 3; l++) {
            const bool rowUsed = l < 2 || o < kOut;
            for (int c = 0; c < 80; c += 16) {
                float v[16];
                if (have) tmem_ld16(tcol(T + gc[l], c), v);
                if (!rowUsed) continue;
                for (int j = 0; j < 16; j++) {
                    const int i = c + j;
                    const float g = have ? v[j] : 0.f;
                    if (i < kHid) P[ow[l] + o * kHid + i] = g;
                    else if (i == kHid) P[ob[l] + o] = g;
                }
            }
        }
    }
    fence_before_sync();
    __syncthreads();
    if (!ok && tid == 0) mbar_wait(&bar, phase, kWaitLimit);
    __syncthreads();
    if (warp == 0) tmem_dealloc(tbase, kTrainCols);
}

// ---------------------------------------------------------------------------
// Parameter maintenance
// ---------------------------------------------------------------------------
// Bias-folded operand row element k of a layer with nin inputs: the weight,
// then the bias as a BF16 pair (hi, lo), then zeros.
__device__ __forceinline__ bf16 folded(const float* master, int ow, int ob, int nin, int o, int k) {
    if (k < nin) return __float2bfloat16_rn(master[ow + o * nin + k]);
    const float b = master[ob + o];
    const bf16 hi = __float2bfloat16_rn(b);
    if (k == nin) return hi;
    if (k == nin + 1) return __float2bfloat16_rn(b - __bfloat162float(hi));
    return __float2bfloat16_rn(0.f);
}

__global__ void k_guide_prepare(const float* master, bf16* blob) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < kBlobAll; e += gridDim.x * blockDim.x) {
        bf16 v;
        if (e < bI2) v = folded(master, oW1, oB1, kIn, (e - bI1) / kInK, (e - bI1) % kInK);
        else if (e < bI3) v = folded(master, oW2, oB2, kHid, (e - bI2) / kHidK, (e - bI2) % kHidK);
        else if (e < bI4) v = folded(master, oW3, oB3, kHid, (e - bI3) / kHidK, (e - bI3) % kHidK);
        else {
            const int o = (e - bI4) / kHidK;
            v = o < kOut ? folded(master, oW4, oB4, kHid, o, (e - bI4) % kHidK) : __float2bfloat16_rn(0.f);
        }
        blob[e] = v;
    }
}

__global__ void k_guide_reduce(const float* partials, int parts, float* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kParams; i += gridDim.x * blockDim.x) {
        float s = 0.f;
        for (int c = 0; c < parts; c++) s += partials[(size_t)c * kParams + i];
        out[i] = s;
    }
}

// The BF16 operand entries of parameter i (its weight, or its bias's hi / lo
// pair) from its FP32 value, as k_guide_prepare writes them.
__device__ __forceinline__ void fold_param(bf16* blob, int i, float x) {
    int base, nin, nk, rel;
    bool bias;
    if (i < oW2) {
        base = bI1; nin = kIn; nk = kInK; bias = i >= oB1; rel = bias ? i - oB1 : i - oW1;
    } else if (i < oW3) {
        base = bI2; nin = kHid; nk = kHidK; bias = i >= oB2; rel = bias ? i - oB2 : i - oW2;
    } else if (i < oW4) {
        base = bI3; nin = kHid; nk = kHidK; bias = i >= oB3; rel = bias ? i - oB3 : i - oW3;
    } else {
        base = bI4; nin = kHid; nk = kHidK; bias = i >= oB4; rel = bias ? i - oB4 : i - oW4;
    }
    if (!bias) {
        blob[base + (rel / nin) * nk + rel % nin] = __float2bfloat16_rn(x);
    } else {
        const bf16 hi = __float2bfloat16_rn(x);
        blob[base + rel * nk + nin] = hi;
        blob[base + rel * nk + nin + 1] = __float2bfloat16_rn(x - __bfloat162float(hi));
    }
}

// One Adam step over the training CTAs' partial gradients. Each block takes
// 32 parameters (one per lane); its warps sum consecutive slices of the
// partials and the slices are added in warp order, a fixed order, so the
// update is the same on every run. The updated parameter's BF16 operand
// entries are written in place (the blob's constant entries were written
// when the guide was made).
constexpr int kAdamWarps = 8;
__global__ void __launch_bounds__(32 * kAdamWarps) k_guide_adam(float* master, float* m, float* v, const float* partials,
                                                                int parts, float lr, float b1, float b2, float eps,
                                                                float c1, float c2, bf16* blob) {
    __shared__ float slice[kAdamWarps][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int i = blockIdx.x * 32 + lane;
    const int per = (parts + kAdamWarps - 1) / kAdamWarps;
    const int cBegin = w * per, cEnd = min(parts, cBegin + per);
    float part = 0.f;
    if (i < kParams)
        for (int c = cBegin; c < cEnd; c++) part += partials[(size_t)c * kParams + i];
    slice[w][lane] = part;
    __syncthreads();
    if (w != 0 || i >= kParams) return;
    float g = 0.f;
#pragma unroll
    for (int k = 0; k < kAdamWarps; k++) g += slice[k][lane];
    const float mi = b1 * m[i] + (1.f - b1) * g;
    const float vi = b2 * v[i] + (1.f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    const float x = master[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    master[i] = x;
    fold_param(blob, i, x);
}

// 1 / (sum of the records' weights), or 0 when the sum is not positive.
__global__ void k_guide_weight_scale(const float* records, int n, const int* count, int offset, int capacity, int stepCap,
                                     float* scale) {
    __shared__ float part[32];
    const int cnt = count ? max(0, min(min(*count, capacity) - offset, stepCap)) : n;
    float s = 0.f;
    for (int i = threadIdx.x; i < cnt; i += blockDim.x) s += records[(size_t)i * MC_GUIDE_RECORD_FLOATS + 9];
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < (int)(blockDim.x >> 5) ? part[threadIdx.x] : 0.f;
        for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
        if (threadIdx.x == 0) *scale = s > 0.f ? 1.0f / s : 0.f;
    }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
struct SplitMix {
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

// He-uniform weights (bound sqrt(6 / fan_in)), the output layer scaled by 0.1,
// zero biases (kappa starts at 1). Anchored lobes start with log kappa 1
// (kappa near e): with every mean near the direction input, the untrained
// mixture is a lobe about as wide as the cosine's.
void init_params(std::vector<float>& p, uint64_t seed, bool anchored) {
    SplitMix r{seed ^ 0x6A09E667F3BCC909ull};
    p.assign(kParams, 0.f);
    auto fill = [&](int off, int out, int in, double gain) {
        double b = std::sqrt(6.0 / in) * gain;
        for (int i = 0; i < out * in; i++) p[off + i] = (float)((2.0 * r.uniform() - 1.0) * b);
    };
    fill(oW1, kHid, kIn, 1.0);
    fill(oW2, kHid, kHid, 1.0);
    fill(oW3, kHid, kHid, 1.0);
    fill(oW4, kOut, kHid, 0.1);
    if (anchored)
        for (int k = 0; k < kLobes; k++) p[oB4 + 32 + k] = 1.0f;
}

// The anchor offset's signed length: the direction input as fed (the normal
// faces the arriving ray), or turned back for the arriving ray's direction.
float anchor_of(const mc_guide* g) {
    if (g->cfg.anchor_lobes == MC_GUIDE_LOBES_RAW) return 0.f;
    return g->cfg.direction_input == MC_GUIDE_DIR_RAY ? -MC_GUIDE_ANCHOR : MC_GUIDE_ANCHOR;
}

// The kernels' opt-in shared-memory sizes, once per context (per device).
mc_status set_attrs(mc_context* ctx) {
    if (ctx->guide_attrs_set) return MC_OK;
    MC_CUDA(cudaFuncSetAttribute(k_guide_train, cudaFuncAttributeMaxDynamicSharedMemorySize, kTrainSmem));
    MC_CUDA(cudaFuncSetAttribute(k_guide_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, kInferSmem));
    ctx->guide_attrs_set = true;
    return MC_OK;
}

void box(const mc_guide* g, float* lo, float* inv) {
    const mc_aabb& b = g->cfg.bounds;
    const float l[3] = {b.lo.x, b.lo.y, b.lo.z}, h[3] = {b.hi.x, b.hi.y, b.hi.z};
    for (int i = 0; i < 3; i++) {
        lo[i] = l[i];
        float ext = h[i] - l[i];
        inv[i] = ext > 0.f ? 1.0f / ext : 1.0f;
    }
}

mc_status prepare(mc_guide* g, cudaStream_t s) {
    k_guide_prepare<<<64, 256, 0, s>>>(g->master, (bf16*)g->blob);
    MC_CUDA(cudaGetLastError());
    return MC_OK;
}

template <class Args>
void fill_box(const mc_guide* g, Args& a) {
    float lo[3], inv[3];
    box(g, lo, inv);
    a.lox = lo[0]; a.loy = lo[1]; a.loz = lo[2];
    a.invx = inv[0]; a.invy = inv[1]; a.invz = inv[2];
}

mc_status launch_train(mc_guide* g, cudaStream_t s, const float* records, int n, const int* count, int offset,
                       int capacity, int stepCap, const float* scale, int* gridOut, float weightCap = 0.f) {
    mc_status st = set_attrs(g->ctx);
    if (st != MC_OK) return st;
    GuideTrainArgs a;
    std::memset(&a, 0, sizeof(a));
    a.blob = (const bf16*)g->blob;
    a.master = g->master;
    fill_box(g, a);
    a.records = records;
    a.n = n;
    a.count = count;
    a.offset = offset;
    a.capacity = capacity;
    a.stepCap = stepCap;
    a.scale = scale;
    a.weightCap = weightCap;
    a.anchor = anchor_of(g);
    a.partials = g->partials;
    a.loss = g->loss;
    a.err = g->ctx->d_error;
    const int sms = g->ctx->sm_count;
    int grid = count ? sms : std::max(1, std::min(sms, (n + kTile - 1) / kTile));
    k_guide_train<<<grid, kTile, kTrainSmem, s>>>(a);
    MC_CUDA(cudaGetLastError());
    *gridOut = grid;
    return MC_OK;
}

mc_status adam_step(mc_guide* g, cudaStream_t s, int parts) {
    const int t = g->steps + 1;
    const float b1 = g->cfg.beta1, b2 = g->cfg.beta2;
    const float c1 = (float)(1.0 - std::pow((double)b1, t)), c2 = (float)(1.0 - std::pow((double)b2, t));
    k_guide_adam<<<(kParams + 31) / 32, 32 * kAdamWarps, 0, s>>>(g->master, g->adam_m, g->adam_v, g->partials, parts,
                                                                 g->cfg.learning_rate, b1, b2, g->cfg.epsilon, c1, c2,
                                                                 (bf16*)g->blob);
    MC_CUDA(cudaGetLastError());
    g->steps = t;
    return MC_OK;
}

mc_status flags_of(mc_context* ctx) {
    int flags = 0;
    MC_CUDA(cudaMemcpyAsync(&flags, ctx->d_error, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    MC_CUDA(cudaStreamSynchronize(ctx->stream));
    return mc::status_from_device_flags(flags);
}

}  // namespace

namespace mc {

mc_status guide_reserve_paths(mc_guide* g, int paths) {
    if (g->mixture_capacity >= paths) return MC_OK;
    cudaFree(g->mixtures);
    cudaFree(g->records);
    cudaFree(g->nee0);
    g->mixtures = g->records = g->nee0 = nullptr;
    g->mixture_capacity = g->record_capacity = 0;
    if (cudaMalloc(&g->mixtures, (size_t)paths * kOut * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&g->records, (size_t)paths * g->cfg.train_vertices * 16 * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&g->nee0, (size_t)paths * 3 * sizeof(float)) != cudaSuccess) {
        cudaGetLastError();
        return set_error(MC_ERR_OOM, "guide: allocation of per-path buffers failed");
    }
    g->mixture_capacity = g->record_capacity = paths;
    return MC_OK;
}

mc_status guide_infer_paths(mc_guide* g, cudaStream_t s, const int* queue, const int* count, int capacity,
                            const float* ox, const float* oy, const float* oz, const float* dx, const float* dy,
                            const float* dz, const float* time, const mc_packed_hit* hits, const mc_triangle_hot* hot,
                            const mc_sphere* spheres, float* mixtures, int stride) {
    mc_status st = set_attrs(g->ctx);
    if (st != MC_OK) return st;
    GuideInferArgs a;
    std::memset(&a, 0, sizeof(a));
    a.blob = (const bf16*)g->blob;
    a.master = g->master;
    fill_box(g, a);
    a.count = count;
    a.capacity = capacity;
    a.queue = queue;
    a.ox = ox; a.oy = oy; a.oz = oz; a.dx = dx; a.dy = dy; a.dz = dz; a.time = time;
    a.hits = hits;
    a.hot = hot;
    a.spheres = spheres;
    a.dirNormal = g->cfg.direction_input == MC_GUIDE_DIR_NORMAL ? 1 : 0;
    a.stride = stride;
    a.anchor = anchor_of(g);
    a.mix = mixtures;
    a.err = g->ctx->d_error;
    k_guide_infer<<<g->ctx->sm_count, kTile * kInferGroups, kInferSmem, s>>>(a);
    MC_CUDA(cudaGetLastError());
    return MC_OK;
}

mc_status guide_reserve_batch(mc_guide* g, int records) {
    if (g->batch_records >= records) return MC_OK;
    float* nb = nullptr;
    if (cudaMalloc(&nb, (size_t)records * MC_GUIDE_RECORD_FLOATS * sizeof(float)) != cudaSuccess) {
        cudaGetLastError();
        return set_error(MC_ERR_OOM, "guide: allocation of the training batch failed");
    }
    cudaFree(g->batch);
    g->batch = nb;
    g->batch_records = records;
    return MC_OK;
}

mc_status guide_reserve_tiles(mc_guide* g, int tiles) {
    if (g->rec_tile_capacity >= tiles) return MC_OK;
    int* nt = nullptr;
    if (cudaMalloc(&nt, (size_t)std::max(tiles, 1) * sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        return set_error(MC_ERR_OOM, "guide: allocation of the record tile counts failed");
    }
    cudaFree(g->rec_tiles);
    g->rec_tiles = nt;
    g->rec_tile_capacity = tiles;
    return MC_OK;
}

mc_status guide_train_device(mc_guide* g, cudaStream_t s, const float* records, const int* count, int capacity, int steps,
                             int stepRecords) {
    const int B = stepRecords > 0 ? std::min(stepRecords, g->cfg.batch_capacity) : g->cfg.batch_capacity;
    for (int i = 0; i < steps; i++) {
        const int off = i * B;
        const float* r = records + (size_t)off * MC_GUIDE_RECORD_FLOATS;
        k_guide_weight_scale<<<1, 1024, 0, s>>>(r, 0, count, off, capacity, B, g->scale);
        MC_CUDA(cudaGetLastError());
        int grid = 0;
        mc_status st = launch_train(g, s, r, 0, count, off, capacity, B, g->scale, &grid, g->cfg.weight_cap);
        if (st != MC_OK) return st;
        if ((st = adam_step(g, s, grid)) != MC_OK) return st;
    }
    return MC_OK;
}

}  // namespace mc

extern "C" {

mc_status mc_guide_create(mc_context* ctx, const mc_guide_config* config, mc_guide** out) {
    if (!ctx || !config || !out) return mc::set_error(MC_ERR_INVALID, "mc_guide_create: null argument");
    *out = nullptr;
    mc_guide* g = new mc_guide();
    g->ctx = ctx;
    g->cfg = *config;
    if (g->cfg.learning_rate <= 0.f) g->cfg.learning_rate = 1e-3f;
    if (g->cfg.beta1 <= 0.f) g->cfg.beta1 = 0.9f;
    if (g->cfg.beta2 <= 0.f) g->cfg.beta2 = 0.999f;
    if (g->cfg.epsilon <= 0.f) g->cfg.epsilon = 1e-8f;
    if (g->cfg.batch_capacity <= 0) g->cfg.batch_capacity = 65536;
    if (g->cfg.train_steps <= 0) g->cfg.train_steps = 1;
    if (!(g->cfg.guide_fraction > 0.f && g->cfg.guide_fraction < 1.f)) g->cfg.guide_fraction = 0.5f;
    // guiding and training at the first bounce only, with anchored lobes,
    // reached plain sampling's error in the least time on the aperture room,
    // from scratch and with a trained guide (inference and guided shading
    // then run for two bounces of the path)
    if (g->cfg.train_vertices <= 0) g->cfg.train_vertices = 1;
    if (g->cfg.guided_depth <= 0) g->cfg.guided_depth = 2;
    if (!(g->cfg.weight_cap >= 0.f)) g->cfg.weight_cap = 0.f;
    if (g->cfg.train_vertices > MC_GUIDE_MAX_TRAIN_VERTICES || g->cfg.direction_input < 0 || g->cfg.direction_input > 1 ||
        g->cfg.anchor_lobes < 0 || g->cfg.anchor_lobes > MC_GUIDE_LOBES_RAW || g->cfg.nee_records < 0 ||
        g->cfg.nee_records > 1) {
        delete g;
        return mc::set_error(MC_ERR_INVALID,
                             "mc_guide_create: train_vertices above %d, unknown direction_input or anchor_lobes, or "
                             "nee_records not 0/1",
                             MC_GUIDE_MAX_TRAIN_VERTICES);
    }
    const size_t P = (size_t)kParams * sizeof(float);
    bool okAlloc = cudaMalloc(&g->master, P) == cudaSuccess && cudaMalloc(&g->adam_m, P) == cudaSuccess &&
                   cudaMalloc(&g->adam_v, P) == cudaSuccess && cudaMalloc(&g->blob, (size_t)kBlobAll * 2) == cudaSuccess &&
                   cudaMalloc(&g->partials, (size_t)ctx->sm_count * P) == cudaSuccess &&
                   cudaMalloc(&g->scale, sizeof(float)) == cudaSuccess && cudaMalloc(&g->loss, sizeof(double)) == cudaSuccess &&
                   cudaMalloc(&g->batch, (size_t)g->cfg.batch_capacity * g->cfg.train_steps * MC_GUIDE_RECORD_FLOATS *
                                             sizeof(float)) == cudaSuccess &&
                   (g->batch_records = g->cfg.batch_capacity * g->cfg.train_steps) > 0 &&
                   cudaMalloc(&g->batch_count, sizeof(int)) == cudaSuccess;
    if (!okAlloc) {
        cudaGetLastError();
        mc_guide_destroy(g);
        return mc::set_error(MC_ERR_OOM, "mc_guide_create: device allocation failed");
    }
    std::vector<float> p;
    init_params(p, g->cfg.seed, g->cfg.anchor_lobes != MC_GUIDE_LOBES_RAW);
    cudaMemcpy(g->master, p.data(), P, cudaMemcpyHostToDevice);
    cudaMemset(g->adam_m, 0, P);
    cudaMemset(g->adam_v, 0, P);
    mc_status st = prepare(g, ctx->stream);
    if (st == MC_OK) {
        cudaError_t e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) st = mc::cuda_error((int)e, "mc_guide_create", __FILE__, __LINE__);
    }
    if (st != MC_OK) {
        mc_guide_destroy(g);
        return st;
    }
    *out = g;
    return MC_OK;
}

// Does not touch the guide's context (which may be gone already): cudaFree
// waits for the device work that uses the buffers.
mc_status mc_guide_destroy(mc_guide* g) {
    if (!g) return MC_OK;
    cudaFree(g->master);
    cudaFree(g->adam_m);
    cudaFree(g->adam_v);
    cudaFree(g->blob);
    cudaFree(g->partials);
    cudaFree(g->scale);
    cudaFree(g->loss);
    cudaFree(g->batch);
    cudaFree(g->batch_count);
    cudaFree(g->rec_tiles);
    cudaFree(g->records);
    cudaFree(g->mixtures);
    cudaFree(g->nee0);
    delete g;
    return MC_OK;
}

mc_status mc_guide_get_params(const mc_guide* g, float* params) {
    if (!g || !params) return mc::set_error(MC_ERR_INVALID, "mc_guide_get_params: null argument");
    MC_CUDA(cudaMemcpyAsync(params, g->master, (size_t)kParams * sizeof(float), cudaMemcpyDeviceToHost, g->ctx->stream));
    MC_CUDA(cudaStreamSynchronize(g->ctx->stream));
    return MC_OK;
}

mc_status mc_guide_set_params(mc_guide* g, const float* params) {
    if (!g || !params) return mc::set_error(MC_ERR_INVALID, "mc_guide_set_params: null argument");
    MC_CUDA(cudaMemcpyAsync(g->master, params, (size_t)kParams * sizeof(float), cudaMemcpyHostToDevice, g->ctx->stream));
    mc_status st = prepare(g, g->ctx->stream);
    if (st != MC_OK) return st;
    MC_CUDA(cudaStreamSynchronize(g->ctx->stream));
    return MC_OK;
}

mc_status mc_guide_infer(mc_guide* g, const float* d_queries, int32_t n, float* d_mixtures) {
    if (!g || n < 0 || (n > 0 && (!d_queries || !d_mixtures))) return mc::set_error(MC_ERR_INVALID, "mc_guide_infer: bad argument");
    if (n == 0) return MC_OK;
    mc_status st = set_attrs(g->ctx);
    if (st != MC_OK) return st;
    mc_context* ctx = g->ctx;
    MC_CUDA(cudaMemsetAsync(ctx->d_error, 0, sizeof(int), ctx->stream));
    GuideInferArgs a;
    std::memset(&a, 0, sizeof(a));
    a.blob = (const bf16*)g->blob;
    a.master = g->master;
    fill_box(g, a);
    a.n = n;
    a.queries = d_queries;
    a.anchor = anchor_of(g);
    a.mix = d_mixtures;
    a.err = ctx->d_error;
    int tiles = (n + kTile - 1) / kTile;
    k_guide_infer<<<std::min((tiles + kInferGroups - 1) / kInferGroups, ctx->sm_count), kTile * kInferGroups, kInferSmem,
                    ctx->stream>>>(a);
    MC_CUDA(cudaGetLastError());
    return flags_of(ctx);
}

mc_status mc_guide_gradient(mc_guide* g, const float* d_records, int32_t n, float* d_grad, double* loss) {
    if (!g || n < 0 || !d_grad || (n > 0 && !d_records)) return mc::set_error(MC_ERR_INVALID, "mc_guide_gradient: bad argument");
    mc_context* ctx = g->ctx;
    MC_CUDA(cudaMemsetAsync(ctx->d_error, 0, sizeof(int), ctx->stream));
    MC_CUDA(cudaMemsetAsync(g->loss, 0, sizeof(double), ctx->stream));
    if (n == 0) {
        MC_CUDA(cudaMemsetAsync(d_grad, 0, (size_t)kParams * sizeof(float), ctx->stream));
        if (loss) *loss = 0.0;
        return flags_of(ctx);
    }
    int grid = 0;
    mc_status st = launch_train(g, ctx->stream, d_records, n, nullptr, 0, 0, 0, nullptr, &grid);
    if (st != MC_OK) return st;
    k_guide_reduce<<<80, 256, 0, ctx->stream>>>(g->partials, grid, d_grad);
    MC_CUDA(cudaGetLastError());
    double l = 0.0;
    MC_CUDA(cudaMemcpyAsync(&l, g->loss, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    st = flags_of(ctx);
    if (loss) *loss = l;
    return st;
}

mc_status mc_guide_train(mc_guide* g, const float* d_records, int32_t n) {
    if (!g || n < 0 || (n > 0 && !d_records)) return mc::set_error(MC_ERR_INVALID, "mc_guide_train: bad argument");
    if (n == 0) return MC_OK;
    mc_context* ctx = g->ctx;
    MC_CUDA(cudaMemsetAsync(ctx->d_error, 0, sizeof(int), ctx->stream));
    MC_CUDA(cudaMemsetAsync(g->loss, 0, sizeof(double), ctx->stream));
    k_guide_weight_scale<<<1, 1024, 0, ctx->stream>>>(d_records, n, nullptr, 0, 0, 0, g->scale);
    MC_CUDA(cudaGetLastError());
    int grid = 0;
    mc_status st = launch_train(g, ctx->stream, d_records, n, nullptr, 0, 0, 0, g->scale, &grid);
    if (st != MC_OK) return st;
    if ((st = adam_step(g, ctx->stream, grid)) != MC_OK) return st;
    return flags_of(ctx);
}

int32_t mc_guide_steps(const mc_guide* g) { return g ? g->steps : 0; }

}  // extern "C"
