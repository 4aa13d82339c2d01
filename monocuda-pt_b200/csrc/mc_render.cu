// mc_render.cu - the wavefront render path on sm_100a, for one scene or a batch.
//
// A wave is one sample of every pixel of every scene in the wave table (a
// single render call is a table of one scene). Per bounce d:
//   trace(d)  persistent kernel: closest hits of the bounce-d extend queue AND
//             the bounce-(d-1) shadow rays, pulled from one work counter by
//             warps that refill idle lanes (PT:3416-3468 extendKernelPersistent
//             + PT:3698-3728 shadowKernel, fused into one launch);
//   shade(d)  grid-stride kernel (PT:3470-3696 shadeKernel) that appends to the
//             next extend queue and to the shadow queue with one atomic per warp.
// Queue sizes never leave the device: every kernel reads its count from the
// per-bounce counter block, and camera/finalize loop over the path count the
// table holds, so a wave is a fixed launch sequence (no host readback per
// bounce as in PT:3816) that is captured once as a CUDA graph and replayed.
// Renders deeper than the counter block (max_depth > 64) are the exception:
// their counters form a ring, the host reads the next bounce's path count
// every 8 bounces to end the wave early, and they are not captured.
//
// Compiled with --use_fast_math like the reference (CMakeLists.txt:94-96).
#include <cuda_runtime.h>
#include <curand_kernel.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "mc_guide.cuh"
#include "mc_internal.h"
#include "mc_rng.cuh"
#include "mc_shade.cuh"
#include "mc_traverse.cuh"
#include "mc_volume.cuh"

#define MC_CUDA(call)                                                                      \
    do {                                                                                   \
        cudaError_t e__ = (call);                                                          \
        if (e__ != cudaSuccess) return mc::cuda_error((int)e__, #call, __FILE__, __LINE__); \
    } while (0)

#define MC_WAVE_MAX_SCENES 128

namespace mc {

// One scene of a wave: its BVH, arrays, camera, image and sample number.
struct SceneGPU {
    const float4* nodes;
    const float4* prims;
    const mc_sphere* spheres;
    const mc_triangle_hot* hot;
    const mc_triangle_cold* cold;
    const mc_light* lights;
    float* accum;
    curandState* xorwow;
    int root;
    int hasMedium;
    int lightCount;
    int W, H;
    // This item's paths in the wave: pathOffset + pixel * pathStride + j for its
    // j = 0..pathStride-1 samples of the wave (sample index `sample` + j):
    // the samples of a pixel are neighbours, so they share warps.
    int pathOffset;
    int pathStride;
    int pixelOffset;  // first pixel of this item among the wave's pixels
    int paths;
    int maxDepth;
    int disableClamp;
    uint32_t sample;
    uint32_t seedLo, seedHi;
    mc_env_map env;
    const int2* envAlias;  // alias table of env (MC_ENV_SAMPLE_ALIAS), else null: CDF inversion
    mc_camera cam;
};

struct WaveTable {
    int nScenes;
    int totalPaths;
    int totalPixels;  // pixels of all items (each holds pathStride paths)
    int pad1;
    SceneGPU scenes[MC_WAVE_MAX_SCENES];
};

namespace {

constexpr unsigned kFull = 0xffffffffu;

MC_D unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

MC_D int scene_of(const WaveTable* tab, const unsigned short* sceneOf, int path) {
    return (tab->nScenes > 1 && sceneOf) ? (int)sceneOf[path] : 0;
}

MC_D int pixel_of(const SceneGPU& S, int path) {
    const int r = path - S.pathOffset;
    return S.pathStride == 1 ? r : r / S.pathStride;
}

MC_D uint32_t sample_of(const SceneGPU& S, int path) {
    return S.pathStride == 1 ? S.sample : S.sample + (uint32_t)((path - S.pathOffset) % S.pathStride);
}

// ---------------------------------------------------------------------------
// Trace: extend rays + shadow rays in one persistent launch.
// ---------------------------------------------------------------------------
struct TraceArgs {
    const WaveTable* tab;
    const unsigned short* sceneOf;
    // single-scene launches: the scene's BVH as kernel parameters (constant bank, no registers)
    TraceScene ts0;
    int medium0;
    const mc_sphere* spheres0;
    const mc_triangle_cold* cold0;
    // extend rays: path indices from queue (identity when null), rays from the path SoA
    const int* queue;
    const int* extCount;
    int extN;
    const float *ox, *oy, *oz, *dx, *dy, *dz, *time;
    mc_packed_hit* hits;
    // shadow rays (PT:3170-3186 layout)
    const int* shCount;
    int shN;
    const float *sox, *soy, *soz, *sdx, *sdy, *sdz, *smax, *scr, *scg, *scb;
    const int* spath;
    float *sr, *sg, *sb;   // per-path sample accumulators
    int* occluded;         // ray-set mode: any-hit result per shadow slot instead of accumulation
    int* work;
    int refill;
    int* err;
    unsigned long long* counts;  // [0] node visits, [1] leaf tests (counting variant)
    int oneShot;                 // plain mode: one ray per thread, no refill
    int stackCap;                // traversal stack entries per lane, <= MC_STACK_CAPACITY (0: all)
    int threads;                 // block size asked for: 128 or 256 (0: 256)
    int queueCap;                // entries the extend and shadow queues hold (counts past it are clamped)
    // launches with gridded media (MC_MEDIUM_GRID): per shadow slot, the
    // distance of each medium crossing and, for back faces, the homogeneous
    // factor or the crossed primitive of a grid; rays that crossed a grid are
    // listed (count in vdefer[0]) for k_ratio_track, which draws their random numbers
    float4* vsegT;
    int4* vsegX;
    int* vmeta;
    int* vdefer;
};

// Warp-reduces the lane counters and adds them to the global pair.
MC_D void flush_counts(const TraceArgs& a, const TravCount& c) {
    unsigned long long v = (unsigned long long)c.visits, l = (unsigned long long)c.leaves;
    for (int off = 16; off > 0; off >>= 1) {
        v += __shfl_xor_sync(0xffffffffu, v, off);
        l += __shfl_xor_sync(0xffffffffu, l, off);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&a.counts[0], v);
        atomicAdd(&a.counts[1], l);
    }
}

enum { RAY_EXTEND = 0, RAY_SHADOW_ANY = 1, RAY_SHADOW_MEDIUM = 2 };

// Finishes one ray. Returns true when the lane is free again. GRID: the
// launch's scenes hold density grids (the crossing bookkeeping for
// k_ratio_track is compiled in only then).
template <int ISECT, bool GRID>
MC_D bool finish_ray(const TraceArgs& a, const TraceScene& ts, const mc_triangle_cold* cold, const mc_sphere* spheres,
                     TravState& s, int step, int kind, int slot, float& T, float& travelled, int& crossings) {
    if (kind == RAY_EXTEND) {
        int type = -1, id = -1, did = 0;
        if (s.hitLeaf >= 0) {
            leaf_identity(ts, s.hitLeaf, type, id);
            did = 1;
        }
        reinterpret_cast<int4*>(a.hits)[slot] = make_int4(__float_as_int(s.tmax), type, id, did);
        return true;
    }
    if (kind == RAY_SHADOW_ANY) {
        if (a.occluded) {
            a.occluded[slot] = step == STEP_OCCLUDED ? 1 : 0;
            return true;
        }
        // PT:3711-3727: unoccluded -> transmittance 1
        if (step != STEP_OCCLUDED) {
            int p = a.spath[slot];
            float tr = 1.0f;
            a.sr[p] += a.scr[slot] * tr;
            a.sg[p] += a.scg[slot] * tr;
            a.sb[p] += a.scb[slot] * tr;
        }
        return true;
    }
    // medium transmittance loop (PT:2874-2898, at most 4 boundary crossings)
    bool done = false;
    bool blocked = false;
    if (s.hitLeaf < 0) {
        done = true;
    } else {
        int type, id;
        leaf_identity(ts, s.hitLeaf, type, id);
        const mc_material* m = type == 1 ? &cold[id].mat : &spheres[id].mat;
        int mtype = m->type;
        float density = m->density;
        if (mtype != MC_MAT_ISOTROPIC) {
            blocked = true;
            done = true;
        } else {
            bool front;
            if (type == 1) {
                const float4* rec = ts.prims + (long long)s.hitLeaf * 3;
                float4 r0 = __ldg(rec), r1 = __ldg(rec + 1), r2 = __ldg(rec + 2);
                V3 v0(r0.x, r0.y, r0.z), v1(r0.w, r1.x, r1.y), v2(r1.z, r1.w, r2.x);
                V3 e1 = v1 - v0;
                V3 e2 = v2 - v0;
                V3 nrm = e1.cross(e2).normalize();
                front = s.r.d.dot(nrm) < 0.0f;
            } else {
                const mc_sphere& sp = spheres[id];
                float tt;
                V3 outward;
                hit_sphere_ref(v3(sp.center), v3(sp.center1), sp.is_moving != 0, sp.radius, s.r.o, s.r.d, s.time, tt, front,
                               outward);
            }
            const int c = GRID ? crossings & 15 : crossings;
            if (!front) {
                if (GRID && m->density_grid) {
                    // ratio tracking draws random numbers: deferred to k_ratio_track.
                    // Ray-set queries (occluded output) draw none and skip the grid.
                    if (a.vsegT) {
                        (&a.vsegX[slot].x)[c] = type == 1 ? id : -1 - id;
                        crossings |= 1 << (4 + c);
                    }
                } else {
                    const float f = expf(-density * s.tmax);
                    T = T * f;
                    if (GRID && a.vsegT) {
                        (&a.vsegX[slot].x)[c] = __float_as_int(f);
                        crossings |= 1 << (8 + c);
                    }
                }
            }
            if (GRID && a.vsegT) (&a.vsegT[slot].x)[c] = s.tmax;
            travelled = travelled + s.tmax;
            V3 hp = s.r.o + s.r.d * s.tmax;
            crossings++;
            float remaining = a.smax[slot] - travelled;
            if ((GRID ? crossings & 15 : crossings) >= 4 || remaining <= 0.0f) {
                done = true;
            } else {
                s.r.o = hp;
                s.tmax = remaining;
                s.hitLeaf = -1;
                s.node = ts.root;
                s.sp = 0;
            }
        }
    }
    if (!done) return false;
    if (a.occluded) {
        a.occluded[slot] = (blocked || !(T > 0.0f)) ? 1 : 0;
        return true;
    }
    if (GRID && (crossings & 0xf0)) {
        // a grid was crossed: k_ratio_track finishes the ray in crossing order
        a.vmeta[slot] = crossings | (blocked ? 1 << 12 : 0);
        a.vdefer[1 + atomicAdd(a.vdefer, 1)] = slot;
        return true;
    }
    if (!blocked && T > 0.0f) {
        int p = a.spath[slot];
        a.sr[p] += a.scr[slot] * T;
        a.sg[p] += a.scg[slot] * T;
        a.sb[p] += a.scb[slot] * T;
    }
    return true;
}

// MED: 1 when some scene of the launch holds a medium, so its shadow rays take
// the closest-hit loop of mediumTransmittance instead of any-hit
// (PT:3711-3720); 2 when some medium also has a density grid.
// BATCH: rays of several scenes share the launch; each lane reads its ray's
// scene from the wave table. A single-scene launch reads the scene from the
// kernel parameters instead, which costs no registers.
// THREADS: 256 (3 resident blocks of up to 85 registers, the default) or 128
// (7 resident blocks of up to 73 registers: 28 warps per SM instead of 24
// when the traversal stack is short enough for 7 blocks' shared memory; a
// variant the autotuner may pick for single-scene launches).
#ifndef MC_TRACE_MIN_BLOCKS
#define MC_TRACE_MIN_BLOCKS 3
#endif
#ifndef MC_TRACE128_MIN_BLOCKS
#define MC_TRACE128_MIN_BLOCKS 7
#endif
constexpr int kTraceThreads = 256;
template <int ISECT, int MED, bool COUNT, int LAY, bool BATCH, int THREADS = kTraceThreads>
__global__ void __launch_bounds__(THREADS, THREADS == 256 ? MC_TRACE_MIN_BLOCKS : MC_TRACE128_MIN_BLOCKS)
    k_trace(TraceArgs a) {
    TravCount cnt;
    const int lane = threadIdx.x & 31;
    const unsigned ltmask = lanemask_lt();
    // a queue that overflowed holds queueCap entries (the producer flagged the overflow)
    const int extCount = a.extCount ? min(*a.extCount, a.queueCap) : a.extN;
    const int shCount = a.shCount ? min(*a.shCount, a.queueCap) : a.shN;
    const int total = extCount + shCount;
#if MC_SMEM_STACK
    extern __shared__ int traceStack[];
    const SharedStack<THREADS> stack{traceStack + threadIdx.x};
#else
    int stackMem[MC_STACK_CAPACITY];
    const LocalStack stack{stackMem};
#endif
    TravState s;
    TraceScene tsLane;
    tsLane.nodes = nullptr;
    tsLane.prims = nullptr;
    tsLane.root = 0;
    const TraceScene& ts = BATCH ? tsLane : a.ts0;
    WatertightRay w;
    w.kx = 0; w.ky = 1; w.kz = 2; w.sx = w.sy = w.sz = 0.f;
    bool has = false, exhausted = total == 0;
    int kind = 0, slot = 0, crossings = 0, sid = 0;
    float T = 1.f, travelled = 0.f;
    while (true) {
        if (!exhausted) {
            unsigned idle = __ballot_sync(kFull, !has);
            int cnt = __popc(idle);
            if (cnt >= a.refill) {
                int leader = __ffs(idle) - 1;
                int base = 0;
                if (a.oneShot) {
                    // plain wavefront (PT:3376-3397): one ray per thread, no refill
                    base = blockIdx.x * blockDim.x + (threadIdx.x & ~31);
                } else {
                    if (lane == leader) base = atomicAdd(a.work, cnt);
                    base = __shfl_sync(kFull, base, leader);
                }
                if (!has) {
                    int q = base + __popc(idle & ltmask);
                    if (q < total) {
                        V3 o, d;
                        float time, tmax;
                        if (q < extCount) {
                            kind = RAY_EXTEND;
                            slot = a.queue ? a.queue[q] : q;
                            if (BATCH) sid = scene_of(a.tab, a.sceneOf, slot);
                            o = V3(a.ox[slot], a.oy[slot], a.oz[slot]);
                            d = V3(a.dx[slot], a.dy[slot], a.dz[slot]);
                            time = a.time[slot];
                            tmax = 1e30f;
                        } else {
                            slot = q - extCount;
                            int path = a.spath ? a.spath[slot] : slot;
                            if (BATCH) sid = scene_of(a.tab, a.sceneOf, path);
                            const bool med = MED != 0 && (BATCH ? a.tab->scenes[sid].hasMedium != 0 : a.medium0 != 0);
                            kind = med ? RAY_SHADOW_MEDIUM : RAY_SHADOW_ANY;
                            o = V3(a.sox[slot], a.soy[slot], a.soz[slot]);
                            d = V3(a.sdx[slot], a.sdy[slot], a.sdz[slot]);
                            time = a.time[path];
                            tmax = a.smax[slot];
                            T = 1.f;
                            travelled = 0.f;
                            crossings = 0;
                        }
                        if (BATCH) {
                            const SceneGPU* S = &a.tab->scenes[sid];
                            tsLane.nodes = S->nodes;
                            tsLane.prims = S->prims;
                            tsLane.root = S->root;
                        }
                        has = true;
                        if (kind == RAY_SHADOW_MEDIUM && tmax <= 0.0f) {
                            // PT:2880-2881: nothing left to traverse, transmittance 1
                            // (no leaf, so the material arrays are not read)
                            s.tmax = tmax;
                            s.hitLeaf = -1;
                            finish_ray<ISECT, MED == 2>(a, ts, nullptr, nullptr, s, STEP_DONE, kind, slot, T, travelled, crossings);
                            has = false;
                        }
                        if (has) {
                            trav_begin(s, o, d, time, tmax, ts.root);
                            if (ISECT == MC_ISECT_WATERTIGHT) w = make_watertight(d);
                        }
                    }
                }
                if (a.oneShot || base + cnt >= total) exhausted = true;
            }
        }
        if (exhausted && __ballot_sync(kFull, has) == 0u) break;
        if (has) {
            int r = (kind == RAY_SHADOW_ANY)
                        ? trav_step_layout<true, ISECT, COUNT, LAY>(ts, s, stack, w, a.err, &cnt, a.stackCap)
                        : trav_step_layout<false, ISECT, COUNT, LAY>(ts, s, stack, w, a.err, &cnt, a.stackCap);
            if (r != STEP_CONTINUE) {
                const mc_triangle_cold* cold = a.cold0;
                const mc_sphere* spheres = a.spheres0;
                if (BATCH && MED != 0 && kind == RAY_SHADOW_MEDIUM) {
                    cold = a.tab->scenes[sid].cold;
                    spheres = a.tab->scenes[sid].spheres;
                }
                if (finish_ray<ISECT, MED == 2>(a, ts, cold, spheres, s, r, kind, slot, T, travelled, crossings)) has = false;
            }
        }
    }
    if (COUNT) flush_counts(a, cnt);
}

// ---------------------------------------------------------------------------
// Shade
// ---------------------------------------------------------------------------
struct ShadeArgs {
    const WaveTable* tab;
    const unsigned short* sceneOf;
    int depth;
    float *ox, *oy, *oz, *dx, *dy, *dz;
    const float* time;
    float *tr, *tg, *tb, *sr, *sg, *sb;
    unsigned char* spec;
    float* pdf;
    uint32_t* draw;
    const mc_packed_hit* hits;
    const int* queue;
    const int* count;
    int* nextQueue;
    int* nextCount;
    float *sox, *soy, *soz, *sdx, *sdy, *sdz, *smax, *scr, *scg, *scb;
    int* spath;
    int* shCount;
    int capacity;
    int* err;
    // guided shading: per-path mixtures of this bounce, the guide's share of
    // the one-sample MIS, the training records of the first recSlots diffuse
    // vertices of each path, and the direction the guide is fed
    const float* mix;
    float guideFrac;
    float* rec;
    int recSlots;
    int dirNormal;
    int mixShare;     // bounce 0 of a single-item pixel-major wave: the pixel's samples read its first path's mixture
    int fold;         // guide directions below the surface are mirrored up (guided_pdf)
    int neeRec;       // the primary vertex's next-event sample also gives a training record
};

// Training record of a diffuse vertex (recSlots per path, slot = depth):
// [0..2] position, [3..5] direction input (face normal or ray direction),
// [6..8] sampled direction, [9] mean throughput that reached the vertex,
// [10] valid (the sampled direction was traced), [11] MIS remainder of the
// emission that direction found, [12] mean sample radiance not carried by
// that direction (everything before the vertex plus its own NEE), [13..15]
// in slot 0 with NEE records: the direction of the vertex's shadow ray (zero
// when it cast none); the light it brought is the primary vertex's NEE buffer.
constexpr int kRecFloats = 16;

// The path whose mixture a path samples: itself, or at a shared bounce 0 the
// first sample of its pixel (the samples of a pixel start with the same
// primary ray; any mixture is a valid proposal, so sharing keeps the estimator
// unbiased whatever the hits).
MC_D int mix_path(const ShadeArgs& a, const SceneGPU& S, int p) {
    return a.mixShare ? p - (p - S.pathOffset) % S.pathStride : p;
}

MC_D float* rec_slot(const ShadeArgs& a, int p, int depth) {
    return a.rec + ((size_t)p * a.recSlots + depth) * kRecFloats;
}

struct ShadeOut {
    bool next;
    bool shadow;
    V3 so, sd, contrib;
    float smax;
};

template <class Rng>
MC_D void rng_load(const ShadeArgs& a, const SceneGPU& S, int p, Rng& rng);
template <>
MC_D void rng_load<PhiloxRng>(const ShadeArgs& a, const SceneGPU& S, int p, PhiloxRng& rng) {
    rng.init(S.seedLo, S.seedHi, sample_of(S, p), (uint32_t)pixel_of(S, p), a.draw[p]);
}
template <>
MC_D void rng_load<XorwowRng>(const ShadeArgs& a, const SceneGPU& S, int p, XorwowRng& rng) {
    rng.st = S.xorwow[pixel_of(S, p)];
}
template <class Rng>
MC_D void rng_store(const ShadeArgs& a, const SceneGPU& S, int p, const Rng& rng);
template <>
MC_D void rng_store<PhiloxRng>(const ShadeArgs& a, const SceneGPU& S, int p, const PhiloxRng& rng) {
    a.draw[p] = rng.draw;
}
template <>
MC_D void rng_store<XorwowRng>(const ShadeArgs& a, const SceneGPU& S, int p, const XorwowRng& rng) {
    S.xorwow[pixel_of(S, p)] = rng.st;
}

struct MatView {
    int type;
    mc_texture albedo;
    V3 emitted;
    float fuzz, ior, density, g;
};

MC_D MatView load_material(const mc_material& m) {
    MatView v;
    v.type = m.type;
    v.albedo = m.albedo;
    v.emitted = v3(m.emitted);
    v.fuzz = m.fuzz;
    v.ior = m.refraction_index;
    v.density = m.density;
    v.g = m.phase_g;
    return v;
}

// Density of the guided direction sampler at a diffuse vertex: the cosine
// lobe with probability 1 - frac, the guide's mixture with probability frac.
// fold: the guide's directions below the surface are folded up (mirrored in
// the tangent plane), so none is lost to a zero BSDF: the guide's density at w
// above the surface is then q(w) + q(w') with w' the mirror image of w, and 0
// below. Without folding a guide direction below the surface ends the path
// (its BSDF is zero): cheaper per sample, noisier while the guide is young.
MC_D float guided_pdf(const float* m, float frac, const V3& n, const V3& w, bool fold) {
    if (!fold) {
        const float c = fmaxf(n.dot(w), 0.0f);
        return (1.0f - frac) * (c / MC_PI) + frac * guide::mixture_pdf(m, w.x, w.y, w.z);
    }
    const float c = n.dot(w);
    if (!(c > 0.0f)) return 0.0f;
    const V3 r = w - n * (2.0f * c);
    return (1.0f - frac) * (c / MC_PI) +
           frac * (guide::mixture_pdf(m, w.x, w.y, w.z) + guide::mixture_pdf(m, r.x, r.y, r.z));
}

// Guided renders: a primary-vertex record must see all the light that arrives
// along its sampled direction. Emission (or environment) found at depth 1 by
// that direction enters the image with its MIS weight w; the part (1 - w) that
// NEE's side of the MIS carries instead is kept in the record's spare slot and
// added to its weight. Without it a broad early guide, whose density is tiny
// next to the light's, would never be pulled toward a small light.
//
// With NEE records (neeRec) the primary vertex's shadow rays are records of
// their own, weighted by NEE's MIS share, so the sampled direction keeps only
// its MIS-weighted share too: the two kinds add up to the incident light.
MC_D void train_remainder(const ShadeArgs& a, int p, int depth, const V3& L, float w) {
    if (w >= 1.0f || depth < 1 || depth > a.recSlots || (a.neeRec && depth == 1)) return;
    float* r = rec_slot(a, p, depth - 1);
    if (r[10] == 0.0f) return;
    r[11] = (L.x + L.y + L.z) * (1.0f / 3.0f) * (1.0f - w);
}

// PT:3470-3696 shadeKernel for one path. GUIDED: diffuse vertices sample the
// next direction by one-sample MIS of the cosine lobe and the guide. ALIAS:
// scenes with an alias table draw environment directions from it; the
// variant without it compiles the reference's CDF sampling on its own, so
// the image-parity path keeps exactly the reference's instruction sequence.
template <class Rng, bool GUIDED, bool ALIAS = false>
MC_D void shade_path(const ShadeArgs& a, const SceneGPU& S, int p, ShadeOut& out) {
    const int depth = a.depth;
    V3 throughput(a.tr[p], a.tg[p], a.tb[p]);
    V3 cs(a.sr[p], a.sg[p], a.sb[p]);
    int4 hraw = reinterpret_cast<const int4*>(a.hits)[p];
    float hitT = __int_as_float(hraw.x);
    int ptype = hraw.y, pidx = hraw.z, didHit = hraw.w;
    const V3 background = v3(S.cam.background);
    const int lightCount = S.lightCount;
    if (GUIDED && a.rec && depth >= 1 && depth <= a.recSlots) {
        // the previous vertex's direction was traced: what the sample holds now
        // (including that vertex's NEE) did not come through it
        float* r = rec_slot(a, p, depth - 1);
        if (r[10] != 0.0f) r[12] = (cs.x + cs.y + cs.z) * (1.0f / 3.0f);
    }
    if (!didHit) {
        V3 missDir(a.dx[p], a.dy[p], a.dz[p]);
        float envW = 1.0f;
        float envProb = env_selection_probability(S.env, lightCount);
        if (!(depth == 0 || a.spec[p] != 0) && envProb > 0.0f)
            envW = power_heuristic(a.pdf[p], envProb * env_direction_pdf(S.env, missDir));
        const V3 envL = throughput * env_radiance(S.env, missDir, background);
        cs = cs + envL * envW;
        if (GUIDED && a.rec) train_remainder(a, p, depth, envL, envW);
        a.sr[p] = cs.x;
        a.sg[p] = cs.y;
        a.sb[p] = cs.z;
        return;
    }
    MatView mat = load_material(ptype == 0 ? S.spheres[pidx].mat : S.cold[pidx].mat);
    V3 inDir(a.dx[p], a.dy[p], a.dz[p]);
    V3 o(a.ox[p], a.oy[p], a.oz[p]);
    float rayTime = a.time[p];
    V3 hitPoint = o + inDir * hitT;
    V3 hitNormal;
    V3 faceNormal;  // geometric normal facing the arriving ray (the guide's direction input)
    bool frontFace;
    float hitU, hitV;
    V3 tv0, tv1, tv2;
    if (ptype == 0) {
        const mc_sphere& sp = S.spheres[pidx];
        V3 c = sphere_center_at(v3(sp.center), v3(sp.center1), sp.is_moving != 0, rayTime);
        V3 outward = (hitPoint - c).normalize();
        frontFace = inDir.dot(outward) < 0.0f;
        hitNormal = frontFace ? outward : -outward;
        faceNormal = hitNormal;
        V2 uv = sphere_uv(outward);
        hitU = uv.x;
        hitV = uv.y;
    } else {
        const mc_triangle_hot& h = S.hot[pidx];
        const mc_triangle_cold& cd = S.cold[pidx];
        tv0 = v3(h.v0); tv1 = v3(h.v1); tv2 = v3(h.v2);
        V3 e1 = tv1 - tv0;
        V3 e2 = tv2 - tv0;
        V3 nrm = e1.cross(e2).normalize();
        frontFace = inDir.dot(nrm) < 0.0f;
        V3 shading = triangle_shading_normal(tv0, tv1, tv2, v3(cd.n0), v3(cd.n1), v3(cd.n2), hitPoint, nrm);
        hitNormal = frontFace ? shading : -shading;
        faceNormal = frontFace ? nrm : -nrm;
        V2 uv = triangle_uv(tv0, tv1, tv2, V2(cd.uv0.x, cd.uv0.y), V2(cd.uv1.x, cd.uv1.y), V2(cd.uv2.x, cd.uv2.y), hitPoint);
        hitU = uv.x;
        hitV = uv.y;
    }
    if (mat.type == MC_MAT_EMISSIVE) {
        bool prevSpec = a.spec[p] != 0;
        float emissionWeight = 1.0f;
        bool fromBsdf = !(depth == 0 || prevSpec);
        if (fromBsdf && ptype == 1) {
            float cosL = fmaxf(fabsf(inDir.dot(hitNormal)), 1e-4f);
            float area = triangle_area(tv0, tv1, tv2);
            float lightPdf = light_solid_angle_pdf((1.0f - env_selection_probability(S.env, lightCount)) / float(lightCount),
                                                   hitT, cosL, area);
            emissionWeight = power_heuristic(a.pdf[p], lightPdf);
        }
        cs = cs + throughput * mat.emitted * emissionWeight;
        if (GUIDED && a.rec) train_remainder(a, p, depth, throughput * mat.emitted, emissionWeight);
        a.sr[p] = cs.x;
        a.sg[p] = cs.y;
        a.sb[p] = cs.z;
        return;
    }
    Rng rng;
    rng_load<Rng>(a, S, p, rng);
    const V3 tPre = throughput;  // what reached this vertex (training records of guided renders)
    V3 scatterOrigin = hitPoint;
    if (mat.type == MC_MAT_ISOTROPIC) {
        float sd;
        const mc_material& M = ptype == 0 ? S.spheres[pidx].mat : S.cold[pidx].mat;
        const mc_volume_grid* grid = static_cast<const mc_volume_grid*>(M.density_grid);
        // a grid in a scene whose flags lack MC_MEDIUM_GRID: its shadow rays were
        // traced without grid bookkeeping
        if (grid && !(S.hasMedium & MC_MEDIUM_GRID)) atomicOr(a.err, MC_DEVERR_INPUT);
        if (frontFace) sd = hitT;  // this hit only enters the medium
        else if (grid) sd = volume_free_flight(grid, mat.density, M.grid_max_density, o, inDir, hitT, rng);  // PT:3562-3564
        else sd = -logf(1.0f - rng.uniform()) / mat.density;
        if (sd >= hitT) {
            a.ox[p] = hitPoint.x;
            a.oy[p] = hitPoint.y;
            a.oz[p] = hitPoint.z;
            out.next = depth + 1 < S.maxDepth;
            rng_store<Rng>(a, S, p, rng);
            return;
        }
        scatterOrigin = o + inDir * sd;
    }
    throughput = throughput * sample_texture(mat.albedo, hitU, hitV);

    float envProb = env_selection_probability(S.env, lightCount);
    if ((mat.type == MC_MAT_LAMBERTIAN || mat.type == MC_MAT_ISOTROPIC) && (lightCount > 0 || envProb > 0.0f)) {
        V3 toLight, lightColor;
        float dist, solidPdf;
        if (envProb > 0.0f && (lightCount == 0 || rng.uniform() < envProb)) {
            float dirPdf;
            if (ALIAS && S.envAlias) toLight = env_sample_alias(S.env, S.envAlias, rng, dirPdf);
            else toLight = env_sample(S.env, rng, dirPdf);
            lightColor = env_radiance(S.env, toLight, V3(0.f, 0.f, 0.f));
            dist = 1e30f;
            solidPdf = envProb * dirPdf;
        } else {
            int li = min((int)(rng.uniform() * lightCount), lightCount - 1);
            const mc_light& L = S.lights[li];
            float sel = (1.0f - envProb) / float(lightCount);
            V3 pt = sample_triangle(v3(L.tri.v0), v3(L.tri.v1), v3(L.tri.v2), rng);
            V3 vec = pt - scatterOrigin;
            dist = vec.length();
            toLight = vec / dist;
            lightColor = v3(L.emitted);
            float cosL = fabsf(v3(L.normal).dot(toLight));
            solidPdf = (cosL > 1e-4f) ? sel * (dist * dist) / (cosL * L.area) : 0.0f;
        }
        bool iso = (mat.type == MC_MAT_ISOTROPIC);
        float cosS = iso ? 1.0f : hitNormal.dot(toLight);
        if (cosS > 0.0f && solidPdf > 0.0f) {
            float phasePdf = hg_phase_pdf(inDir.dot(toLight), mat.g);
            float scatterPdf = iso ? phasePdf : lambertian_cosine_pdf(cosS);
            if (GUIDED && !iso && mat.type == MC_MAT_LAMBERTIAN)
                scatterPdf = guided_pdf(a.mix + (size_t)mix_path(a, S, p) * guide::kOut, a.guideFrac, hitNormal, toLight, a.fold != 0);
            float scatterValue = iso ? phasePdf : cosS / MC_PI;
            float neeW = power_heuristic(solidPdf, scatterPdf);
            V3 contribution = throughput * lightColor * (scatterValue / solidPdf) * neeW;
            out.shadow = true;
            out.so = scatterOrigin;
            out.sd = toLight;
            out.smax = dist * 0.999f;
            out.contrib = contribution;
        }
        if (GUIDED && a.rec && a.neeRec && depth == 0 && mat.type == MC_MAT_LAMBERTIAN) {
            // the vertex fields of slot 0 (the sampled direction's record writes
            // the same values), and the shadow ray's direction
            float* r = rec_slot(a, p, 0);
            const V3 din = a.dirNormal ? faceNormal : inDir;
            r[0] = scatterOrigin.x; r[1] = scatterOrigin.y; r[2] = scatterOrigin.z;
            r[3] = din.x; r[4] = din.y; r[5] = din.z;
            r[9] = (tPre.x + tPre.y + tPre.z) * (1.0f / 3.0f);
            if (out.shadow) {
                r[13] = toLight.x; r[14] = toLight.y; r[15] = toLight.z;
            }
        }
    }
    bool survives = true;
    if (depth > 3) {
        float maxC = fmaxf(throughput.x, fmaxf(throughput.y, throughput.z));
        float cont = fminf(maxC, S.cam.rr_cap);
        if (rng.uniform() > cont) survives = false;
        else throughput = throughput / cont;
    }
    float guidedPdf = 0.0f;
    V3 nd;
    if (survives) {
        V3 rayDir(a.dx[p], a.dy[p], a.dz[p]);
        switch (mat.type) {
            case MC_MAT_CONDUCTOR: {
                V3 refl = specular_scatter(rayDir, hitNormal);
                nd = (refl + random_unit_vector(rng) * mat.fuzz).normalize();
                break;
            }
            case MC_MAT_DIELECTRIC: {
                float ratio = frontFace ? 1.0f / mat.ior : mat.ior;
                nd = dielectric_scatter(rayDir, hitNormal, ratio, rng);
                break;
            }
            case MC_MAT_ISOTROPIC: nd = hg_scatter(inDir, mat.g, rng); break;
            case MC_MAT_LAMBERTIAN:
            default:
                if (GUIDED) {
                    const float* m = a.mix + (size_t)mix_path(a, S, p) * guide::kOut;
                    if (rng.uniform() < a.guideFrac) {
                        float u0 = rng.uniform(), u1 = rng.uniform(), u2 = rng.uniform();
                        float d3[3];
                        guide::mixture_sample(m, u0, u1, u2, d3);
                        nd = V3(d3[0], d3[1], d3[2]);
                        const float below = nd.dot(hitNormal);
                        if (a.fold && below < 0.0f) nd = nd - hitNormal * (2.0f * below);  // folded up (guided_pdf)
                    } else {
                        nd = lambertian_scatter(hitNormal, rng);
                    }
                    const float c = nd.dot(hitNormal);
                    if (!(c > 0.0f)) {
                        survives = false;  // below the surface: the BSDF is zero
                        break;
                    }
                    guidedPdf = guided_pdf(m, a.guideFrac, hitNormal, nd, a.fold != 0);
                    throughput = throughput * ((c / MC_PI) / guidedPdf);
                    if (a.rec && depth < a.recSlots && depth + 1 < S.maxDepth) {
                        // the direction is traced next: a training record of this vertex
                        float* r = rec_slot(a, p, depth);
                        const V3 din = a.dirNormal ? faceNormal : inDir;
                        r[0] = scatterOrigin.x; r[1] = scatterOrigin.y; r[2] = scatterOrigin.z;
                        r[3] = din.x; r[4] = din.y; r[5] = din.z;
                        r[6] = nd.x; r[7] = nd.y; r[8] = nd.z;
                        r[9] = (tPre.x + tPre.y + tPre.z) * (1.0f / 3.0f);
                        r[10] = 1.0f;
                    }
                } else {
                    nd = lambertian_scatter(hitNormal, rng);
                }
                break;
        }
    }
    if (survives) {
        a.ox[p] = scatterOrigin.x;
        a.oy[p] = scatterOrigin.y;
        a.oz[p] = scatterOrigin.z;
        a.dx[p] = nd.x;
        a.dy[p] = nd.y;
        a.dz[p] = nd.z;
        a.tr[p] = throughput.x;
        a.tg[p] = throughput.y;
        a.tb[p] = throughput.z;
        a.spec[p] = (mat.type != MC_MAT_LAMBERTIAN && mat.type != MC_MAT_ISOTROPIC) ? 1 : 0;
        a.pdf[p] = (mat.type == MC_MAT_ISOTROPIC) ? hg_phase_pdf(inDir.dot(nd), mat.g)
                   : (GUIDED && mat.type == MC_MAT_LAMBERTIAN) ? guidedPdf
                                                               : lambertian_cosine_pdf(fmaxf(nd.dot(hitNormal), 0.0f));
        out.next = depth + 1 < S.maxDepth;  // the scene's max depth ends the path (PT:3793)
    }
    rng_store<Rng>(a, S, p, rng);
}

// Warp-aggregated append: one atomicAdd per warp, slots in lane order.
MC_D int warp_reserve(bool want, int* counter, unsigned ltmask) {
    unsigned m = __ballot_sync(kFull, want);
    if (m == 0u) return -1;
    int lane = threadIdx.x & 31;
    int leader = __ffs(m) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(counter, __popc(m));
    base = __shfl_sync(kFull, base, leader);
    return want ? base + __popc(m & ltmask) : -1;
}

// Shading waits on scattered loads (hit, material, light, texture), so its
// residency trades warps against spills: 3 resident blocks (80 registers, no
// spills in the Philox variants) render the benchmark 0.6 % faster than 4
// blocks of 64 registers (118-byte spills), which beat 2 blocks of 113 by 5 %.
// Guided shading: 3 blocks (80 registers, 46-byte spills) take 8 % less time
// than 2 blocks of 127.
#ifndef MC_SHADE_BLOCKS
#define MC_SHADE_BLOCKS 3
#endif
#ifndef MC_GUIDED_SHADE_BLOCKS
#define MC_GUIDED_SHADE_BLOCKS 3
#endif
template <class Rng, bool GUIDED, bool ALIAS = false>
__global__ void __launch_bounds__(256, GUIDED ? MC_GUIDED_SHADE_BLOCKS : MC_SHADE_BLOCKS) k_shade(ShadeArgs a) {
    const unsigned ltmask = lanemask_lt();
    const int count = min(*a.count, a.capacity);
    for (int base = blockIdx.x * blockDim.x; base < count; base += gridDim.x * blockDim.x) {
        int q = base + threadIdx.x;
        ShadeOut out;
        out.next = false;
        out.shadow = false;
        int p = -1;
        if (q < count) {
            p = a.queue[q];
            const SceneGPU& S = a.tab->scenes[scene_of(a.tab, a.sceneOf, p)];
            if (GUIDED && a.rec && a.depth == 0) {
                // every path of the wave passes here first: its record slots start empty
                for (int k = 0; k < a.recSlots; k++) {
                    float* r = rec_slot(a, p, k);
                    r[10] = 0.0f;
                    r[11] = 0.0f;
                    r[12] = 0.0f;
                }
                if (a.neeRec) {
                    float* r = rec_slot(a, p, 0);
                    r[13] = 0.0f;
                    r[14] = 0.0f;
                    r[15] = 0.0f;
                }
            }
            shade_path<Rng, GUIDED, ALIAS>(a, S, p, out);
        }
        int ns = warp_reserve(out.shadow, a.shCount, ltmask);
        if (out.shadow) {
            if (ns < a.capacity) {
                a.sox[ns] = out.so.x;
                a.soy[ns] = out.so.y;
                a.soz[ns] = out.so.z;
                a.sdx[ns] = out.sd.x;
                a.sdy[ns] = out.sd.y;
                a.sdz[ns] = out.sd.z;
                a.smax[ns] = out.smax;
                a.scr[ns] = out.contrib.x;
                a.scg[ns] = out.contrib.y;
                a.scb[ns] = out.contrib.z;
                a.spath[ns] = p;
            } else {
                atomicOr(a.err, MC_DEVERR_QUEUE);
            }
        }
        int nn = warp_reserve(out.next, a.nextCount, ltmask);
        if (out.next) {
            if (nn < a.capacity) a.nextQueue[nn] = p;
            else atomicOr(a.err, MC_DEVERR_QUEUE);
        }
    }
}

// ---------------------------------------------------------------------------
// Camera rays (PT:3342-3374) and per-sample finalize (PT:3740-3755)
// ---------------------------------------------------------------------------
struct CameraArgs {
    const WaveTable* tab;
    unsigned short* sceneOf;
    float *ox, *oy, *oz, *dx, *dy, *dz, *time;
    float *tr, *tg, *tb, *sr, *sg, *sb;
    unsigned char* spec;
    float* pdf;
    uint32_t* draw;
    int* queue;
    int* count;
    int capacity;  // entries the extend queue holds
    int* err;
};

MC_D int find_scene(const WaveTable* tab, int p) {
    int lo = 0, hi = tab->nScenes - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (tab->scenes[mid].pathOffset <= p) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

MC_D void camera_rng(const SceneGPU& S, int pixel, uint32_t sample, PhiloxRng& rng) { rng.init(S.seedLo, S.seedHi, sample, (uint32_t)pixel, 0u); }
MC_D void camera_rng(const SceneGPU& S, int pixel, uint32_t, XorwowRng& rng) { rng.st = S.xorwow[pixel]; }
MC_D void camera_rng_store(const CameraArgs& a, const SceneGPU& S, int p, int pixel, const PhiloxRng& rng) { a.draw[p] = rng.draw; }
MC_D void camera_rng_store(const CameraArgs& a, const SceneGPU& S, int p, int pixel, const XorwowRng& rng) { S.xorwow[pixel] = rng.st; }

template <class Rng>
__global__ void k_camera(CameraArgs a) {
    const int total = a.tab->totalPaths;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *a.count = total;
        if (total > a.capacity) atomicOr(a.err, MC_DEVERR_QUEUE);  // the trace reads the first `capacity`
    }
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < total; p += gridDim.x * blockDim.x) {
        int sid = a.tab->nScenes > 1 ? find_scene(a.tab, p) : 0;
        const SceneGPU& S = a.tab->scenes[sid];
        if (a.tab->nScenes > 1 && a.sceneOf) a.sceneOf[p] = (unsigned short)sid;
        int pixel = pixel_of(S, p);
        int px = pixel % S.W, py = pixel / S.W;
        Rng rng;
        camera_rng(S, pixel, sample_of(S, p), rng);
        V3 o, d;
        float t;
        camera_ray(S.cam, px, py, rng, o, d, t);
        a.ox[p] = o.x; a.oy[p] = o.y; a.oz[p] = o.z;
        a.dx[p] = d.x; a.dy[p] = d.y; a.dz[p] = d.z;
        a.time[p] = t;
        a.tr[p] = 1.0f; a.tg[p] = 1.0f; a.tb[p] = 1.0f;
        a.sr[p] = 0.0f; a.sg[p] = 0.0f; a.sb[p] = 0.0f;
        a.spec[p] = 1;
        a.pdf[p] = 1.0f;
        a.queue[p] = p;
        camera_rng_store(a, S, p, pixel, rng);
    }
}

MC_D int find_scene_by_pixel(const WaveTable* tab, int u) {
    int lo = 0, hi = tab->nScenes - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (tab->scenes[mid].pixelOffset <= u) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// PT:3740-3755 per-sample clamp and accumulation. One thread per pixel adds the
// pixel's samples of the wave in sample order, as consecutive one-sample waves
// would, so the sums are the same to the bit.
__global__ void k_finalize(const WaveTable* tab, const float* sr, const float* sg, const float* sb) {
    const int pixels = tab->totalPixels;
    for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < pixels; u += gridDim.x * blockDim.x) {
        const SceneGPU& S = tab->scenes[tab->nScenes > 1 ? find_scene_by_pixel(tab, u) : 0];
        const int q = u - S.pixelOffset;
        float* acc = S.accum + (size_t)q * 3;
        float a0 = acc[0], a1 = acc[1], a2 = acc[2];
        for (int j = 0; j < S.pathStride; j++) {
            const int p = S.pathOffset + q * S.pathStride + j;
            V3 s(sr[p], sg[p], sb[p]);
            float bright = fmaxf(s.x, fmaxf(s.y, s.z));
            const float maxBright = 10.0f;
            if (!S.disableClamp && bright > maxBright) s = s * (maxBright / bright);
            a0 = a0 + s.x;
            a1 = a1 + s.y;
            a2 = a2 + s.z;
        }
        acc[0] = a0;
        acc[1] = a1;
        acc[2] = a2;
    }
}

// A guided wave's training batch holds its records in (sample, vertex,
// pixel) order: sample j of every pixel before sample j + 1 of any, so that
// an Adam step on a pixel count of records sees about one sample of the
// whole image, as with one sample per wave, and the batch (and so the
// trained guide) is the same on every run. Entry v of that order is vertex
// slot (v / P) % R of sample v / (P R) of wave pixel v % P (P pixels, R record
// slots per path). When the wave has more entries than the batch holds, only
// entries with (pixel + sample R + slot + recPhase) % recStride == 0 are kept,
// the host rotating recPhase between waves, so that records come from the
// whole image and every depth. A kept entry is a record when its slot holds a
// record of positive, finite weight: the mean sample radiance that arrived
// through the sampled direction (the sample minus what it held before that
// direction was traced, plus the MIS remainder of emission the direction
// found) over the mean throughput that reached the vertex. The primary
// vertex's NEE goes to its own buffer, so the sample holds none of it. With
// NEE records each path has one more slot after its R vertex slots: the
// primary vertex's shadow ray, a record when it reached light (its NEE buffer
// over the throughput that reached the vertex; the sampled direction's record
// then carries no MIS remainder).
constexpr int kRecThreads = 256;
constexpr int kRecTileChunks = 8;
constexpr int kRecTile = kRecThreads * kRecTileChunks;  // entries per tile

struct RecSource {
    const float *sr, *sg, *sb;  // the wave's samples
    const float *nr, *ng, *nb;  // the primary vertices' NEE
    const float* rec;
    int recSlots;               // vertex slots per path
    int neeRec;                 // 1: one more slot per path, the primary vertex's shadow ray
};

// dirOff: where the record's direction sits in its slot (6 for a sampled
// direction, 13 for a shadow ray).
MC_D bool rec_entry(const WaveTable* tab, long long v, const RecSource& src, int recStride, int recPhase,
                    const float** out, float* weight, int* dirOff) {
    const int slots = src.recSlots + src.neeRec;
    const int pixels = tab->totalPixels;
    const long long js = v / pixels;
    const int u = (int)(v - js * pixels);
    const int j = (int)(js / slots);
    const int k = (int)(js - (long long)j * slots);
    if ((u + j * slots + k + recPhase) % recStride != 0) return false;
    const SceneGPU& S = tab->scenes[tab->nScenes > 1 ? find_scene_by_pixel(tab, u) : 0];
    if (j >= S.pathStride) return false;
    const int p = S.pathOffset + (u - S.pixelOffset) * S.pathStride + j;
    float w;
    const float* r;
    if (k == src.recSlots) {
        r = src.rec + (size_t)p * src.recSlots * kRecFloats;
        if (!(r[9] > 0.0f) || (r[13] == 0.0f && r[14] == 0.0f && r[15] == 0.0f)) return false;
        w = (src.nr[p] + src.ng[p] + src.nb[p]) * (1.0f / 3.0f) / r[9];
        *dirOff = 13;
    } else {
        r = src.rec + ((size_t)p * src.recSlots + k) * kRecFloats;
        if (r[10] == 0.0f || !(r[9] > 0.0f)) return false;
        w = ((src.sr[p] + src.sg[p] + src.sb[p]) * (1.0f / 3.0f) - r[12] + r[11]) / r[9];
        *dirOff = 6;
    }
    *out = r;
    *weight = w;
    return w > 0.0f && w < 1e30f;
}

// Guided renders (one scene, one or more images): the sample plus the primary
// vertex's NEE goes to the image, and each tile of the wave's training entries
// (`entries` of them, none when not training) counts its records.
__global__ void __launch_bounds__(kRecThreads) k_finalize_guided(const WaveTable* tab, const unsigned short* sceneOf,
                                                                 const float* sr, const float* sg, const float* sb,
                                                                 const float* nr, const float* ng, const float* nb,
                                                                 const float* rec, int* tileCounts, long long entries,
                                                                 int recSlots, int neeRec, int recStride, int recPhase) {
    // the image: each pixel adds its samples of the wave in sample order
    const int pixels = tab->totalPixels;
    for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < pixels; u += gridDim.x * blockDim.x) {
        const SceneGPU& S = tab->scenes[tab->nScenes > 1 ? find_scene_by_pixel(tab, u) : 0];
        const int q = u - S.pixelOffset;
        float* acc = S.accum + (size_t)q * 3;
        float a0 = acc[0], a1 = acc[1], a2 = acc[2];
        for (int j = 0; j < S.pathStride; j++) {
            const int p = S.pathOffset + q * S.pathStride + j;
            V3 s = V3(sr[p], sg[p], sb[p]) + V3(nr[p], ng[p], nb[p]);
            float bright = fmaxf(s.x, fmaxf(s.y, s.z));
            if (!S.disableClamp && bright > 10.0f) s = s * (10.0f / bright);
            a0 = a0 + s.x;
            a1 = a1 + s.y;
            a2 = a2 + s.z;
        }
        acc[0] = a0;
        acc[1] = a1;
        acc[2] = a2;
    }
    if (!rec) return;
    const RecSource src{sr, sg, sb, nr, ng, nb, rec, recSlots, neeRec};
    // the training records: each tile's count (k_rec_scan and k_rec_write place them)
    const int tiles = (int)((entries + kRecTile - 1) / kRecTile);
    for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
        int c = 0;
        for (int i = 0; i < kRecTileChunks; i++) {
            const long long v = (long long)t * kRecTile + i * kRecThreads + threadIdx.x;
            const float* r;
            float w;
            int dirOff;
            c += __syncthreads_count(v < entries && rec_entry(tab, v, src, recStride, recPhase, &r, &w, &dirOff));
        }
        if (threadIdx.x == 0) tileCounts[t] = c;
    }
}

// Exclusive scan of the wave's tile counts by one block of 1024 threads: each
// tile's first batch slot, and the wave's record count in *batchCount.
__global__ void __launch_bounds__(1024) k_rec_scan(int* tileCounts, int tiles, int* batchCount) {
    __shared__ int warpSums[32];
    __shared__ int carry;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < tiles; base += 1024) {
        const int t = base + threadIdx.x;
        const int c = t < tiles ? tileCounts[t] : 0;
        int x = c;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(kFull, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warpSums[wid] = x;
        __syncthreads();
        if (wid == 0) {
            int s = warpSums[lane];
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(kFull, s, o);
                if (lane >= o) s += y;
            }
            warpSums[lane] = s;
        }
        __syncthreads();
        const int before = carry + (wid > 0 ? warpSums[wid - 1] : 0) + x - c;
        if (t < tiles) tileCounts[t] = before;
        __syncthreads();
        if (threadIdx.x == 1023) carry = before + c;
        __syncthreads();
    }
    if (threadIdx.x == 0) *batchCount = carry;
}

// Writes each kept record to its slot in (sample, pixel) order: the tile's
// first slot (k_rec_scan) plus the kept entries before it in the tile.
__global__ void __launch_bounds__(kRecThreads) k_rec_write(const WaveTable* tab, const RecSource src, const int* tileFirst,
                                                           long long entries, int recStride, int recPhase,
                                                           float* batch, int capacity) {
    __shared__ int warpCount[kRecThreads / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const unsigned ltmask = lanemask_lt();
    const int tiles = (int)((entries + kRecTile - 1) / kRecTile);
    for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
        int next = tileFirst[t];
        for (int i = 0; i < kRecTileChunks; i++) {
            const long long v = (long long)t * kRecTile + i * kRecThreads + threadIdx.x;
            const float* r = nullptr;
            float w = 0.f;
            int dirOff = 6;
            const bool e = v < entries && rec_entry(tab, v, src, recStride, recPhase, &r, &w, &dirOff);
            const unsigned m = __ballot_sync(kFull, e);
            if (lane == 0) warpCount[wid] = __popc(m);
            __syncthreads();
            int before = next, all = 0;
            for (int k = 0; k < kRecThreads / 32; k++) {
                const int c = warpCount[k];
                if (k < wid) before += c;
                all += c;
            }
            const int slot = before + __popc(m & ltmask);
            if (e && slot < capacity) {
                float* b = batch + (size_t)slot * MC_GUIDE_RECORD_FLOATS;
                for (int k = 0; k < 6; k++) b[k] = r[k];
                for (int k = 0; k < 3; k++) b[6 + k] = r[dirOff + k];
                b[9] = w;
            }
            next += all;
            __syncthreads();
        }
    }
}

// Finishes the shadow rays that crossed a density grid (k_trace lists them),
// as mediumTransmittance does (PT:2874-2898): each crossing's segment starts
// where the previous one ended; a back face multiplies the transmittance, in
// crossing order, by its homogeneous factor or by ratio tracking through the
// grid on the path's random numbers, which are stored back (PT:3712-3716).
// Runs after the trace launch and before the next shade, the reference's
// order of draws (shade, then shadow, then the next shade).
struct RatioArgs {
    const float4* segT;
    const int4* segX;
    const int* meta;
    const int* list;       // [0] count, then shadow slots
    float *sr, *sg, *sb;   // the sample accumulators of the trace launch
};

template <class Rng>
__global__ void __launch_bounds__(256) k_ratio_track(ShadeArgs a, RatioArgs v) {
    const int n = min(v.list[0], a.capacity);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int slot = v.list[1 + i];
        const int p = a.spath[slot];
        const SceneGPU& S = a.tab->scenes[scene_of(a.tab, a.sceneOf, p)];
        const int meta = v.meta[slot];
        const float4 ts = v.segT[slot];
        const int4 xs = v.segX[slot];
        V3 o(a.sox[slot], a.soy[slot], a.soz[slot]);
        const V3 d(a.sdx[slot], a.sdy[slot], a.sdz[slot]);
        Rng rng;
        rng_load<Rng>(a, S, p, rng);
        float T = 1.0f;
        const int count = meta & 15;
        for (int c = 0; c < count; c++) {
            const float t = (&ts.x)[c];
            const int x = (&xs.x)[c];
            if (meta & (1 << (4 + c))) {
                const mc_material& m = x >= 0 ? S.cold[x].mat : S.spheres[-1 - x].mat;
                T = T * volume_transmittance(static_cast<const mc_volume_grid*>(m.density_grid), m.density,
                                             m.grid_max_density, o, d, t, rng);
            } else if (meta & (1 << (8 + c))) {
                T = T * __int_as_float(x);
            }
            o = o + d * t;
        }
        rng_store<Rng>(a, S, p, rng);
        if (!(meta & (1 << 12)) && T > 0.0f) {
            v.sr[p] += a.scr[slot] * T;
            v.sg[p] += a.scg[slot] * T;
            v.sb[p] += a.scb[slot] * T;
        }
    }
}

// Renders deeper than the counter block (max_depth > MC_MAX_DEPTH_STATS) use
// its MC_MAX_DEPTH_STATS + 1 slots as a ring: bounce d's counters live in
// slot d % kRingSlots. Before bounce d + kRingSlots reuses a slot, its counts
// go to the statistics (the last bucket holds depth 63 and deeper) and it is
// cleared.
constexpr int kRingSlots = MC_MAX_DEPTH_STATS + 1;

__global__ void k_recycle_slot(int* slot, int depth, long long* stats) {
    if (threadIdx.x != 0) return;
    const int b = min(depth, MC_MAX_DEPTH_STATS - 1);
    stats[b] += slot[0];
    stats[MC_MAX_DEPTH_STATS + b] += slot[1];
    for (int k = 0; k < MC_COUNTERS_PER_DEPTH; k++) slot[k] = 0;
}

// The depths [lo, hi) still in the ring at the end of a deep wave.
__global__ void k_accumulate_ring(const int* counters, int lo, int hi, long long* stats) {
    if (threadIdx.x != 0) return;  // one thread: several depths share the last bucket
    for (int d = lo; d < hi; d++) {
        const int* c = counters + (d % kRingSlots) * MC_COUNTERS_PER_DEPTH;
        const int b = min(d, MC_MAX_DEPTH_STATS - 1);
        stats[b] += c[0];
        stats[MC_MAX_DEPTH_STATS + b] += c[1];
    }
}

__global__ void k_accumulate_counts(const int* counters, int maxDepth, long long* stats) {
    int d = threadIdx.x;
    if (d >= maxDepth || d >= MC_MAX_DEPTH_STATS) return;
    stats[d] += counters[d * MC_COUNTERS_PER_DEPTH + 0];
    stats[MC_MAX_DEPTH_STATS + d] += counters[d * MC_COUNTERS_PER_DEPTH + 1];
}

__global__ void k_init_xorwow(curandState* states, int pixels, unsigned long long seed) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < pixels) curand_init(seed, p, 0, &states[p]);  // PT:2870
}

int occupancy_blocks(const void* fn, int sms, size_t smem = 0, int threads = 256) {
    int per = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, threads, smem);
    if (per < 1) per = 1;
    return per * sms;
}

typedef void (*TraceKernel)(TraceArgs);

// [batch][layout][count][medium kind][isect]
#define MC_TKM(C, L, B)                                                                                   \
    {{k_trace<0, 0, C, L, B>, k_trace<1, 0, C, L, B>}, {k_trace<0, 1, C, L, B>, k_trace<1, 1, C, L, B>}, \
     {k_trace<0, 2, C, L, B>, k_trace<1, 2, C, L, B>}}
#define MC_TK(L, B) {MC_TKM(false, L, B), MC_TKM(true, L, B)}
// medium: 0 none, 1 homogeneous media only, 2 media with density grids
TraceKernel trace_kernel(bool batch, int layout, bool count, int medium, int isect) {
    static const TraceKernel table[2][3][2][3][2] = {{MC_TK(0, false), MC_TK(1, false), MC_TK(2, false)},
                                                     {MC_TK(0, true), MC_TK(1, true), MC_TK(2, true)}};
    return table[batch ? 1 : 0][layout][count ? 1 : 0][medium][isect ? 1 : 0];
}
// The 128-thread variant, compiled for launches of the reference intersector
// without counters or density grids; [batch][layout][medium kind].
#define MC_TK128(B)                                                                                     \
    {{k_trace<0, 0, false, 0, B, 128>, k_trace<0, 1, false, 0, B, 128>},                                \
     {k_trace<0, 0, false, 1, B, 128>, k_trace<0, 1, false, 1, B, 128>},                                \
     {k_trace<0, 0, false, 2, B, 128>, k_trace<0, 1, false, 2, B, 128>}}
TraceKernel trace_kernel_128(bool batch, int layout, int medium) {
    static const TraceKernel table[2][3][2] = {MC_TK128(false), MC_TK128(true)};
    return table[batch ? 1 : 0][layout][medium];
}

// Persistent: one wave of resident blocks (SMs x resident blocks per SM) that
// pull rays from the work counter. Plain (PT:3376-3397): the same kernel with
// one ray per thread and no refill, over plainBlocks blocks; sharing the kernel
// keeps the per-ray arithmetic identical between the two modes. A launch is a
// batch launch when it carries a per-path scene map.
void launch_trace(mc_context* ctx, cudaStream_t stream, const TraceArgs& t0, int layout, int medium, int isect,
                  bool persistent, int plainBlocks, bool count = false) {
    TraceArgs t = t0;
    t.oneShot = persistent ? 0 : 1;
    if (t.stackCap <= 0 || t.stackCap > MC_STACK_CAPACITY) t.stackCap = MC_STACK_CAPACITY;
    const bool batch = t.sceneOf != nullptr;
    // the 128-thread variant where it is compiled, else 256 threads
    const bool small = t.threads == 128 && !count && isect == 0 && medium < 2;
    const int threads = small ? 128 : kTraceThreads;
    // the shared-memory stack holds stackCap entries per lane
    const int smem = MC_SMEM_STACK ? threads * t.stackCap * (int)sizeof(int) : 0;
    TraceKernel fn = small ? trace_kernel_128(batch, layout, medium) : trace_kernel(batch, layout, count, medium, isect);
    const int key = medium + 3 * (isect ? 1 : 0) + 6 * (count ? 1 : 0) + 12 * (batch ? 1 : 0) + 24 * layout +
                    72 * (small ? 1 : 0);  // < 144
    if (smem > 48 * 1024 && ctx->trace_smem_attr[key] < smem) {
        cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        ctx->trace_smem_attr[key] = smem;
    }
    // plain launches: one ray per thread (plainBlocks counts 256-thread blocks)
    int blocks = std::max(1, small ? 2 * plainBlocks : plainBlocks);
    if (persistent) {
        if (!ctx->trace_blocks[key] || ctx->trace_blocks_smem[key] != smem) {
            ctx->trace_blocks[key] = occupancy_blocks((const void*)fn, ctx->sm_count, smem, threads);
            ctx->trace_blocks_smem[key] = smem;
        }
        blocks = ctx->trace_blocks[key];
    }
    fn<<<blocks, threads, smem, stream>>>(t);
}

}  // namespace

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
mc_status ensure_wave(mc_context* ctx, int capacity) {
    WaveBuffers& w = ctx->wave;
    if (w.capacity >= capacity && w.block.ptr) return MC_OK;
    size_t n = (size_t)capacity;
    // 28 float/int arrays of n entries (path state 15 + draw + 2 queues + shadow 11),
    // one byte array and the 16-byte hit records; every array 256-byte aligned.
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    size_t f4 = al(n * 4);
    size_t total = 29 * f4 + al(n) + al(n * 16);
    mc_status st = devbuf_reserve(w.block, total);
    if (st != MC_OK) return st;
    char* b = (char*)w.block.ptr;
    auto take = [&](size_t bytes) { char* r = b; b += bytes; return r; };
    w.ox = (float*)take(f4); w.oy = (float*)take(f4); w.oz = (float*)take(f4);
    w.dx = (float*)take(f4); w.dy = (float*)take(f4); w.dz = (float*)take(f4);
    w.time = (float*)take(f4);
    w.tr = (float*)take(f4); w.tg = (float*)take(f4); w.tb = (float*)take(f4);
    w.sr = (float*)take(f4); w.sg = (float*)take(f4); w.sb = (float*)take(f4);
    w.pdf = (float*)take(f4);
    w.draw = (uint32_t*)take(f4);
    w.queue[0] = (int*)take(f4); w.queue[1] = (int*)take(f4);
    w.sox = (float*)take(f4); w.soy = (float*)take(f4); w.soz = (float*)take(f4);
    w.sdx = (float*)take(f4); w.sdy = (float*)take(f4); w.sdz = (float*)take(f4);
    w.smax = (float*)take(f4);
    w.scr = (float*)take(f4); w.scg = (float*)take(f4); w.scb = (float*)take(f4);
    w.spath = (int*)take(f4);
    take(f4);  // spare
    w.spec = (unsigned char*)take(al(n));
    w.hits = (mc_packed_hit*)take(al(n * 16));
    w.capacity = capacity;
    // the graph captured for the old buffers is stale
    if (ctx->graph_exec) {
        cudaGraphExecDestroy((cudaGraphExec_t)ctx->graph_exec);
        ctx->graph_exec = nullptr;
        std::memset(ctx->graph_key, 0, sizeof(ctx->graph_key));
    }
    return MC_OK;
}

static mc_status ensure_tables(mc_context* ctx, int capacity) {
    if (!ctx->d_table) {
        MC_CUDA(cudaMalloc(&ctx->d_table, sizeof(WaveTable)));
        MC_CUDA(cudaMallocHost(&ctx->h_tables, 4 * sizeof(WaveTable)));
        for (int i = 0; i < 4; i++) MC_CUDA(cudaEventCreateWithFlags((cudaEvent_t*)&ctx->table_events[i], cudaEventDisableTiming));
    }
    if (ctx->scene_of_capacity < capacity) {
        if (ctx->scene_of) cudaFree(ctx->scene_of);
        ctx->scene_of = nullptr;
        ctx->scene_of_capacity = 0;
        MC_CUDA(cudaMalloc(&ctx->scene_of, (size_t)capacity * sizeof(unsigned short)));
        ctx->scene_of_capacity = capacity;
        if (ctx->graph_exec) {
            cudaGraphExecDestroy((cudaGraphExec_t)ctx->graph_exec);
            ctx->graph_exec = nullptr;
            std::memset(ctx->graph_key, 0, sizeof(ctx->graph_key));
        }
    }
    return MC_OK;
}

// A pinned host table that no copy in flight reads any more.
static WaveTable* next_host_table(mc_context* ctx, int* slot) {
    int s = ctx->table_slot;
    ctx->table_slot = (s + 1) & 3;
    cudaEventSynchronize((cudaEvent_t)ctx->table_events[s]);
    *slot = s;
    return (WaveTable*)ctx->h_tables + s;
}

mc_status rng_reset(mc_context* ctx, int pixels, unsigned long long seed) {
    if (ctx->rng_pixels < pixels || !ctx->rng_states) {
        if (ctx->rng_states) cudaFree(ctx->rng_states);
        ctx->rng_states = nullptr;
        ctx->rng_pixels = 0;
        if (cudaMalloc(&ctx->rng_states, (size_t)pixels * sizeof(curandState)) != cudaSuccess) {
            cudaGetLastError();
            return set_error(MC_ERR_OOM, "rng: allocation of %d states failed", pixels);
        }
        ctx->rng_pixels = pixels;
    }
    k_init_xorwow<<<(pixels + 255) / 256, 256, 0, ctx->stream>>>((curandState*)ctx->rng_states, pixels, seed);
    MC_CUDA(cudaGetLastError());
    ctx->rng_seed = seed;
    ctx->rng_ready = true;
    return MC_OK;
}

static SceneGPU scene_gpu(mc_context* ctx, const mc_bvh* shared, const WaveItem& it, int pathOffset, uint32_t sample) {
    SceneGPU g;
    std::memset(&g, 0, sizeof(g));
    const mc_bvh* bvh = it.bvh ? it.bvh : shared;
    const bool wide = bvh->layout != MC_BVH_LAYOUT_BINARY;
    g.nodes = (const float4*)(wide ? bvh->wide_nodes : bvh->nodes);
    g.prims = (const float4*)(wide ? bvh->wide_prims : bvh->prims);
    g.root = it.root;
    g.spheres = it.view->spheres;
    g.hot = it.view->tri_hot;
    g.cold = it.view->tri_cold;
    g.lights = it.view->lights;
    g.lightCount = it.view->light_count;
    g.hasMedium = it.view->has_medium;
    g.env = it.view->env;
    g.envAlias = it.p->env_sampling == MC_ENV_SAMPLE_ALIAS ? static_cast<const int2*>(env_alias_table(g.env)) : nullptr;
    g.cam = it.p->camera;
    g.W = it.p->width;
    g.H = it.p->height;
    g.pathOffset = pathOffset;
    g.pathStride = 1;
    g.paths = it.p->width * it.p->height;
    g.maxDepth = it.p->max_depth;
    g.disableClamp = it.p->disable_clamp;
    g.sample = sample;
    g.seedLo = (uint32_t)it.p->seed;
    g.seedHi = (uint32_t)(it.p->seed >> 32);
    g.accum = it.accum;
    g.xorwow = (curandState*)ctx->rng_states;
    return g;
}

// The scene of a single-scene trace launch, passed as kernel parameters.
static void set_single_scene(TraceArgs& t, const mc_bvh* bvh, int root, const mc_scene_view* v) {
    const bool wide = bvh->layout != MC_BVH_LAYOUT_BINARY;
    t.ts0.nodes = (const float4*)(wide ? bvh->wide_nodes : bvh->nodes);
    t.ts0.prims = (const float4*)(wide ? bvh->wide_prims : bvh->prims);
    t.ts0.root = root;
    t.medium0 = v->has_medium;
    t.cold0 = v->tri_cold;
    t.spheres0 = v->spheres;
}

// Runs waves until every item has rendered its spp samples. All items share
// the launch configuration of items[0] (layout, persistence, RNG, intersector).
mc_status run_waves(mc_context* ctx, const mc_bvh* bvh, const WaveItem* items, int n, bool useGraph, bool timed,
                    RenderTiming* tm, mc_guide* guide, bool train) {
    const mc_render_params& p0 = *items[0].p;
    const int layout = bvh->layout;
    const bool philox = p0.rng == MC_RNG_PHILOX;
    const int isect = p0.intersector;
    const bool persistent = p0.persistent != 0;
    const bool countVisits = (p0.instrument & 1) != 0;
    const bool timeTrace = (p0.instrument & 2) != 0;
    int capacity = 0, maxD = 0, waves = 0;
    bool medium = false, grid = false;
    auto item_spw = [&](int i) { return std::max(1, std::min(items[i].spw, std::max(1, items[i].p->spp))); };
    auto item_waves = [&](int i) { return (items[i].p->spp + item_spw(i) - 1) / item_spw(i); };
    // every item on one scene: single-scene trace launches
    bool sameScene = true;
    for (int i = 0; i < n; i++) {
        capacity += items[i].p->width * items[i].p->height * item_spw(i);
        maxD = std::max(maxD, items[i].p->max_depth);
        waves = std::max(waves, item_waves(i));
        medium = medium || items[i].view->has_medium;
        grid = grid || (items[i].view->has_medium & MC_MEDIUM_GRID) != 0;
        if (items[i].view != items[0].view || items[i].bvh != items[0].bvh || items[i].root != items[0].root)
            sameScene = false;
    }
    mc_status st;
    if ((st = ensure_wave(ctx, capacity)) != MC_OK) return st;
    if ((st = ensure_tables(ctx, capacity)) != MC_OK) return st;
    WaveBuffers& w = ctx->wave;
    // deeper than the counter block: ring slots, a stop once a bounce has no
    // paths left (read back every 8 bounces), no graph
    const bool deep = maxD > MC_MAX_DEPTH_STATS;
    if (timeTrace || countVisits || guide || deep) useGraph = false;
    cudaStream_t stream = ctx->stream;
    if (useGraph && !stream) {
        if (!ctx->own_stream) MC_CUDA(cudaStreamCreate(&ctx->own_stream));
        stream = ctx->own_stream;
    }
    int* shadeBlocks = ctx->shade_blocks;
    if (!shadeBlocks[0]) shadeBlocks[0] = occupancy_blocks((const void*)k_shade<PhiloxRng, false>, ctx->sm_count);
    if (!shadeBlocks[1]) shadeBlocks[1] = occupancy_blocks((const void*)k_shade<XorwowRng, false>, ctx->sm_count);
    if (guide && !shadeBlocks[2]) shadeBlocks[2] = occupancy_blocks((const void*)k_shade<PhiloxRng, true>, ctx->sm_count);
    const int guidedBlocks = shadeBlocks[2];
    // the alias-sampling shade variant when some item asked for it (items
    // without an alias table still sample by CDF inside it)
    bool alias = false;
    for (int i = 0; i < n; i++) alias = alias || items[i].p->env_sampling == MC_ENV_SAMPLE_ALIAS;
    const int plainBlocks = (2 * capacity + 255) / 256;
    const int loopBlocks = ctx->sm_count * 8;
    const WaveTable* dtab = (const WaveTable*)ctx->d_table;
    unsigned short* sceneOf = n > 1 ? ctx->scene_of : nullptr;

    CameraArgs ca;
    ca.tab = dtab;
    ca.sceneOf = sceneOf;
    ca.ox = w.ox; ca.oy = w.oy; ca.oz = w.oz; ca.dx = w.dx; ca.dy = w.dy; ca.dz = w.dz; ca.time = w.time;
    ca.tr = w.tr; ca.tg = w.tg; ca.tb = w.tb; ca.sr = w.sr; ca.sg = w.sg; ca.sb = w.sb;
    ca.spec = w.spec; ca.pdf = w.pdf; ca.draw = w.draw; ca.queue = w.queue[0];
    ca.count = ctx->d_counters;
    // entries each queue may hold: the wave's paths, or fewer when the caller
    // asked for a smaller queue (the excess is dropped and reported as overflow)
    const int queueCap = p0.queue_capacity > 0 ? std::min(p0.queue_capacity, capacity) : capacity;
    ca.capacity = queueCap;
    ca.err = ctx->d_error;

    ShadeArgs sa;
    std::memset(&sa, 0, sizeof(sa));
    sa.tab = dtab;
    sa.sceneOf = sceneOf;
    sa.ox = w.ox; sa.oy = w.oy; sa.oz = w.oz; sa.dx = w.dx; sa.dy = w.dy; sa.dz = w.dz; sa.time = w.time;
    sa.tr = w.tr; sa.tg = w.tg; sa.tb = w.tb; sa.sr = w.sr; sa.sg = w.sg; sa.sb = w.sb;
    sa.spec = w.spec; sa.pdf = w.pdf; sa.draw = w.draw; sa.hits = w.hits;
    sa.sox = w.sox; sa.soy = w.soy; sa.soz = w.soz; sa.sdx = w.sdx; sa.sdy = w.sdy; sa.sdz = w.sdz; sa.smax = w.smax;
    sa.scr = w.scr; sa.scg = w.scg; sa.scb = w.scb; sa.spath = w.spath;
    sa.capacity = queueCap;
    sa.err = ctx->d_error;

    TraceArgs ta;
    std::memset(&ta, 0, sizeof(ta));
    ta.tab = dtab;
    ta.sceneOf = sceneOf;
    ta.ox = w.ox; ta.oy = w.oy; ta.oz = w.oz; ta.dx = w.dx; ta.dy = w.dy; ta.dz = w.dz; ta.time = w.time;
    ta.hits = w.hits;
    ta.sox = w.sox; ta.soy = w.soy; ta.soz = w.soz; ta.sdx = w.sdx; ta.sdy = w.sdy; ta.sdz = w.sdz; ta.smax = w.smax;
    ta.scr = w.scr; ta.scg = w.scg; ta.scb = w.scb; ta.spath = w.spath;
    ta.sr = w.sr; ta.sg = w.sg; ta.sb = w.sb;
    ta.err = ctx->d_error;
    ta.queueCap = queueCap;
    ta.stackCap = p0.stack_entries;
    ta.threads = p0.trace_threads;
    if (ta.threads == 0 && ta.stackCap == 0) {
        // by default the 128-thread shape (7 blocks per SM) when every tree of
        // the wave is a greedy 4-wide collapse whose stack need (3 entries per
        // level, rounded up to 8) lets 7 blocks share an SM; the image does
        // not depend on it
        int levels = 0;
        for (int i = 0; i < n && levels >= 0; i++) {
            const mc_bvh* b = items[i].bvh ? items[i].bvh : bvh;
            levels = (b->layout == MC_BVH_LAYOUT_BINARY || b->wide_levels <= 0) ? -1 : std::max(levels, b->wide_levels);
        }
        const int need = levels > 0 ? ((3 * levels + 7) / 8) * 8 : 999;
        if (need <= 56 && isect == MC_ISECT_REFERENCE) {
            ta.threads = 128;
            ta.stackCap = need;
        }
    }
    ta.refill = (p0.refill_threshold > 0 && p0.refill_threshold <= 32) ? p0.refill_threshold : 8;  // PT:3400
    if (countVisits) ta.counts = (unsigned long long*)(ctx->d_stats + 2 * MC_MAX_DEPTH_STATS);
    if (sameScene) {
        // one scene: the trace reads it from kernel parameters
        set_single_scene(ta, items[0].bvh ? items[0].bvh : bvh, items[0].root, items[0].view);
        ta.sceneOf = nullptr;
    }

    RatioArgs ra;
    std::memset(&ra, 0, sizeof(ra));
    if (grid) {
        // per shadow slot: crossing distances (float4), factors / grid primitives
        // (int4), the crossing mask (int); then the list of deferred slots
        const size_t cap = (size_t)capacity;
        if ((st = devbuf_reserve(ctx->volume, cap * 36 + (cap + 1) * sizeof(int))) != MC_OK) return st;
        char* base = (char*)ctx->volume.ptr;
        ta.vsegT = (float4*)base;
        ta.vsegX = (int4*)(base + cap * 16);
        ta.vmeta = (int*)(base + cap * 32);
        ta.vdefer = (int*)(base + cap * 36);
        ra.segT = ta.vsegT;
        ra.segX = ta.vsegX;
        ra.meta = ta.vmeta;
        ra.list = ta.vdefer;
    }

    int* C = ctx->d_counters;
    const size_t counterBytes = (size_t)(MC_MAX_DEPTH_STATS + 1) * MC_COUNTERS_PER_DEPTH * sizeof(int);
    std::vector<cudaEvent_t> traceEvents;
    // instrument bit 1: CUDA events around each timed launch, by phase
    // (0 trace, 1 shade, 2 guide inference, 3 guide training with its record compaction)
    std::vector<int> phaseOf;
    auto phaseBegin = [&](int phase) {
        if (!timeTrace) return;
        cudaEvent_t e;
        cudaEventCreate(&e);
        cudaEventRecord(e, stream);
        traceEvents.push_back(e);
        phaseOf.push_back(phase);
    };
    auto phaseEnd = [&]() {
        if (!timeTrace) return;
        cudaEvent_t e;
        cudaEventCreate(&e);
        cudaEventRecord(e, stream);
        traceEvents.push_back(e);
    };
    int launches = 0;
    int waveR = 1;       // samples per pixel in the current wave (the most any item traces)
    int wavePixels = 0;  // pixels of the current wave
    int recStride = 1, recPhase = 0;  // training-record subsampling of the current wave
    if (guide && train) {
        int maxR = 1;
        for (int i = 0; i < n; i++) maxR = std::max(maxR, item_spw(i));
        if ((st = guide_reserve_batch(guide, guide->cfg.batch_capacity * guide->cfg.train_steps * maxR)) != MC_OK) return st;
        long long pixelsAll = 0;
        for (int i = 0; i < n; i++) pixelsAll += (long long)items[i].p->width * items[i].p->height;
        const long long slotsAll = guide->cfg.train_vertices + (guide->cfg.nee_records ? 1 : 0);
        if ((st = guide_reserve_tiles(guide, (int)((pixelsAll * maxR * slotsAll + kRecTile - 1) / kRecTile))) != MC_OK)
            return st;
    }
    // the launch sequence of one wave (device table already holds the wave)
    float* nee0[3] = {nullptr, nullptr, nullptr};
    if (guide) {
        nee0[0] = guide->nee0;
        nee0[1] = guide->nee0 + capacity;
        nee0[2] = guide->nee0 + 2 * (size_t)capacity;
    }
    auto slot = [&](int d) { return C + (deep ? d % kRingSlots : d) * MC_COUNTERS_PER_DEPTH; };
    // guided renders: the bounces that sample the guide (training needs the
    // record slots' next bounce in the guided shade as well)
    int guidedDepth = guide ? guide->cfg.guided_depth : 0;
    // one image per wave: at bounce 0 the samples of a pixel (neighbouring
    // paths, the same primary ray) share one inference
    const bool shareMix = guide && n == 1;
    if (guide && train && guidedDepth > 0) guidedDepth = std::max(guidedDepth, guide->cfg.train_vertices + 1);
    auto enqueue_wave = [&]() -> mc_status {
        MC_CUDA(cudaMemsetAsync(C, 0, counterBytes, stream));
        if (guide) {
            MC_CUDA(cudaMemsetAsync(guide->nee0, 0, (size_t)capacity * 3 * sizeof(float), stream));
            MC_CUDA(cudaMemsetAsync(guide->batch_count, 0, sizeof(int), stream));
        }
        if (philox) k_camera<PhiloxRng><<<loopBlocks, 256, 0, stream>>>(ca);
        else k_camera<XorwowRng><<<loopBlocks, 256, 0, stream>>>(ca);
        launches++;
        int dEnd = maxD;
        bool stop = false;
        for (int d = 0; d <= maxD; d++) {
            const bool last = d == maxD || stop;  // shadow rays of the previous bounce only
            TraceArgs t = ta;
            if (!last) {
                t.queue = w.queue[d & 1];
                t.extCount = slot(d) + 0;
            } else {
                t.queue = nullptr;
                t.extCount = nullptr;
                t.extN = 0;
            }
            if (d > 0) t.shCount = slot(d - 1) + 1;
            else { t.shCount = nullptr; t.shN = 0; }
            t.work = slot(d) + 2;
            if (guide && d == 1) {
                // the primary vertex's NEE lands apart from the sample so that
                // its training records see only the light through the sampled direction
                t.sr = nee0[0]; t.sg = nee0[1]; t.sb = nee0[2];
            }
            if (grid && d > 0) MC_CUDA(cudaMemsetAsync(ta.vdefer, 0, sizeof(int), stream));
            phaseBegin(0);
            launch_trace(ctx, stream, t, layout, grid ? 2 : medium ? 1 : 0, isect, persistent, plainBlocks, countVisits);
            phaseEnd();
            launches++;
            if (grid && d > 0) {
                RatioArgs r = ra;
                r.sr = t.sr; r.sg = t.sg; r.sb = t.sb;
                if (philox || guide) k_ratio_track<PhiloxRng><<<loopBlocks, 256, 0, stream>>>(sa, r);
                else k_ratio_track<XorwowRng><<<loopBlocks, 256, 0, stream>>>(sa, r);
                launches++;
            }
            if (last) {
                dEnd = d;
                break;
            }
            // bounces past the guided depth shade with the cosine lobe alone: no inference
            const bool guidedBounce = guide && (guidedDepth == 0 || d < guidedDepth);
            if (guidedBounce) {
                phaseBegin(2);
                mc_status gs = guide_infer_paths(guide, stream, w.queue[d & 1], slot(d) + 0, capacity,
                                                 w.ox, w.oy, w.oz, w.dx, w.dy, w.dz, w.time, w.hits,
                                                 items[0].view->tri_hot, items[0].view->spheres, guide->mixtures,
                                                 d == 0 && shareMix ? waveR : 1);
                phaseEnd();
                if (gs != MC_OK) return gs;
                launches++;
            }
            if (deep && d + 1 >= kRingSlots) {
                // slot(d + 1) still holds bounce d + 1 - kRingSlots (last read by its
                // shadow rays' trace, long done): count it and clear it for shade(d)
                k_recycle_slot<<<1, 32, 0, stream>>>(slot(d + 1), d + 1 - kRingSlots, ctx->d_stats);
                launches++;
            }
            ShadeArgs sd = sa;
            sd.depth = d;
            sd.queue = w.queue[d & 1];
            sd.count = slot(d) + 0;
            sd.nextQueue = w.queue[(d + 1) & 1];
            sd.nextCount = slot(d + 1) + 0;
            sd.shCount = slot(d) + 1;
            if (guidedBounce) {
                sd.mix = guide->mixtures;
                sd.guideFrac = guide->cfg.guide_fraction;
                sd.rec = train ? guide->records : nullptr;
                sd.recSlots = guide->cfg.train_vertices;
                sd.dirNormal = guide->cfg.direction_input == MC_GUIDE_DIR_NORMAL ? 1 : 0;
                sd.mixShare = d == 0 && shareMix ? 1 : 0;
                sd.fold = guide->cfg.fold_below ? 1 : 0;
                sd.neeRec = train && guide->cfg.nee_records ? 1 : 0;
                phaseBegin(1);
                if (alias) k_shade<PhiloxRng, true, true><<<guidedBlocks, 256, 0, stream>>>(sd);
                else k_shade<PhiloxRng, true><<<guidedBlocks, 256, 0, stream>>>(sd);
                phaseEnd();
            } else if (philox) {
                phaseBegin(1);
                if (alias) k_shade<PhiloxRng, false, true><<<shadeBlocks[0], 256, 0, stream>>>(sd);
                else k_shade<PhiloxRng, false><<<shadeBlocks[0], 256, 0, stream>>>(sd);
                phaseEnd();
            } else {
                phaseBegin(1);
                if (alias) k_shade<XorwowRng, false, true><<<shadeBlocks[1], 256, 0, stream>>>(sd);
                else k_shade<XorwowRng, false><<<shadeBlocks[1], 256, 0, stream>>>(sd);
                phaseEnd();
            }
            launches++;
            if (deep && (d & 7) == 7 && d + 1 < maxD) {
                // no path continues: the next bounce traces the last shadow rays only
                int next = 0;
                MC_CUDA(cudaMemcpyAsync(&next, slot(d + 1), sizeof(int), cudaMemcpyDeviceToHost, stream));
                MC_CUDA(cudaStreamSynchronize(stream));
                stop = next == 0;
            }
        }
        if (guide) {
            const int slots = guide->cfg.train_vertices;
            const int neeRec = guide->cfg.nee_records ? 1 : 0;
            const long long entries = train ? (long long)(slots + neeRec) * waveR * wavePixels : 0;
            k_finalize_guided<<<loopBlocks, kRecThreads, 0, stream>>>(dtab, sceneOf, w.sr, w.sg, w.sb, nee0[0], nee0[1],
                                                                      nee0[2], train ? guide->records : nullptr,
                                                                      guide->rec_tiles, entries, slots, neeRec,
                                                                      recStride, recPhase);
            if (train) {
                phaseBegin(3);
                const int tiles = (int)((entries + kRecTile - 1) / kRecTile);
                const RecSource src{w.sr, w.sg, w.sb, nee0[0], nee0[1], nee0[2], guide->records, slots, neeRec};
                k_rec_scan<<<1, 1024, 0, stream>>>(guide->rec_tiles, tiles, guide->batch_count);
                k_rec_write<<<loopBlocks, kRecThreads, 0, stream>>>(dtab, src, guide->rec_tiles, entries, recStride,
                                                                    recPhase, guide->batch,
                                                                    guide->cfg.batch_capacity * guide->cfg.train_steps *
                                                                        waveR);
                phaseEnd();
                launches += 2;
            }
        } else {
            k_finalize<<<loopBlocks, 256, 0, stream>>>(dtab, w.sr, w.sg, w.sb);
        }
        if (deep) k_accumulate_ring<<<1, 32, 0, stream>>>(C, std::max(0, dEnd - (kRingSlots - 1)), dEnd, ctx->d_stats);
        else k_accumulate_counts<<<1, 64, 0, stream>>>(C, maxD, ctx->d_stats);
        launches += 2;
        if (guide && train) {
            // as many Adam steps per sample, on as many records each, as with
            // one sample per wave (a sample holds at most a record per pixel)
            phaseBegin(3);
            mc_status gs = guide_train_device(guide, stream, guide->batch, guide->batch_count,
                                              guide->cfg.batch_capacity * guide->cfg.train_steps * waveR,
                                              guide->cfg.train_steps * waveR, wavePixels);
            phaseEnd();
            if (gs != MC_OK) return gs;
            launches += 4 * guide->cfg.train_steps * waveR;
        }
        MC_CUDA(cudaGetLastError());
        return MC_OK;
    };

    cudaGraphExec_t exec = nullptr;
    if (useGraph) {
        // the captured launches bake in these values; any change needs a new capture
        unsigned long long key[16] = {(unsigned long long)(uintptr_t)stream,
                                      (unsigned long long)capacity,
                                      (unsigned long long)maxD,
                                      (unsigned long long)((layout << 6) | (medium ? 2 : 0) | (philox ? 4 : 0) |
                                                           (persistent ? 8 : 0) | (n > 1 ? 16 : 0) |
                                                           (sameScene ? 32 : 0) | (grid ? 1024 : 0)),
                                      (unsigned long long)isect,
                                      (unsigned long long)ta.refill,
                                      (unsigned long long)(uintptr_t)ta.ts0.nodes,
                                      (unsigned long long)(uintptr_t)ta.ts0.prims,
                                      (unsigned long long)ta.ts0.root,
                                      (unsigned long long)ta.medium0,
                                      (unsigned long long)(uintptr_t)ta.cold0,
                                      (unsigned long long)(uintptr_t)ta.spheres0,
                                      (unsigned long long)(uintptr_t)w.block.ptr,
                                      (unsigned long long)(uintptr_t)sceneOf,
                                      (unsigned long long)(uintptr_t)dtab,
                                      1ull};
        if (ctx->graph_exec && std::memcmp(ctx->graph_key, key, sizeof(key)) == 0) {
            exec = (cudaGraphExec_t)ctx->graph_exec;
        } else {
            if (ctx->graph_exec) cudaGraphExecDestroy((cudaGraphExec_t)ctx->graph_exec);
            ctx->graph_exec = nullptr;
            std::memset(ctx->graph_key, 0, sizeof(ctx->graph_key));
            cudaGraph_t graph;
            MC_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
            mc_status cs = enqueue_wave();
            cudaError_t ce = cudaStreamEndCapture(stream, &graph);
            if (cs != MC_OK) return cs;
            if (ce != cudaSuccess) return cuda_error((int)ce, "cudaStreamEndCapture", __FILE__, __LINE__);
            ce = cudaGraphInstantiate(&exec, graph, 0);
            cudaGraphDestroy(graph);
            if (ce != cudaSuccess) return cuda_error((int)ce, "cudaGraphInstantiate", __FILE__, __LINE__);
            ctx->graph_exec = exec;
            std::memcpy(ctx->graph_key, key, sizeof(key));
        }
        launches = 0;
    }

    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (timed) {
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, stream);
    }
    int perWave = 0;
    for (int wv = 0; wv < waves; wv++) {
        int slot;
        WaveTable* h = next_host_table(ctx, &slot);
        int off = 0, pix = 0, k = 0;
        waveR = 1;
        for (int i = 0; i < n; i++) {
            if (item_waves(i) <= wv) continue;
            const int m = item_spw(i);
            const int r = std::min(m, items[i].p->spp - wv * m);
            waveR = std::max(waveR, r);
            const int px = items[i].p->width * items[i].p->height;
            SceneGPU g = scene_gpu(ctx, bvh, items[i], off, (uint32_t)(items[i].p->first_sample + wv * m));
            g.pathStride = r;
            g.pixelOffset = pix;
            h->scenes[k++] = g;
            off += px * r;
            pix += px;
        }
        h->nScenes = k;
        h->totalPaths = off;
        h->totalPixels = pix;
        wavePixels = pix;
        if (guide) {
            const long long cap = (long long)guide->cfg.batch_capacity * guide->cfg.train_steps * waveR;
            const long long entries = (long long)(guide->cfg.train_vertices + (guide->cfg.nee_records ? 1 : 0)) * off;
            recStride = (int)std::max(1ll, (entries + cap - 1) / cap);
            recPhase = wv % recStride;
        }
        h->pad1 = 0;
        size_t bytes = offsetof(WaveTable, scenes) + (size_t)std::max(k, 1) * sizeof(SceneGPU);
        MC_CUDA(cudaMemcpyAsync(ctx->d_table, h, bytes, cudaMemcpyHostToDevice, stream));
        MC_CUDA(cudaEventRecord((cudaEvent_t)ctx->table_events[slot], stream));
        if (useGraph) {
            MC_CUDA(cudaGraphLaunch(exec, stream));
            perWave = 3 + 2 * maxD + (grid ? maxD : 0);
        } else {
            if ((st = enqueue_wave()) != MC_OK) return st;
        }
    }
    if (useGraph) launches = perWave * waves;
    if (timed) {
        cudaEventRecord(e1, stream);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (tm) tm->ms = ms;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    if (tm) tm->kernel_launches = launches;
    if (!traceEvents.empty()) {
        cudaEventSynchronize(traceEvents.back());
        for (size_t i = 0; i + 1 < traceEvents.size(); i += 2) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, traceEvents[i], traceEvents[i + 1]);
            if (!tm) continue;
            switch (phaseOf[i / 2]) {
                case 0: tm->trace_ms += ms; tm->trace_launches++; break;
                case 1: tm->shade_ms += ms; break;
                case 2: tm->infer_ms += ms; break;
                default: tm->train_ms += ms; break;
            }
        }
        for (cudaEvent_t e : traceEvents) cudaEventDestroy(e);
    }
    if (stream != ctx->stream) MC_CUDA(cudaStreamSynchronize(stream));
    return MC_OK;
}

mc_status check_params(const mc_render_params* p, const mc_scene_view* v) {
    if (!p || !v) return set_error(MC_ERR_INVALID, "render: null argument");
    if (p->width <= 0 || p->height <= 0) return set_error(MC_ERR_INVALID, "render: width and height must be positive");
    if ((long long)p->width * p->height >= (1ll << 30)) return set_error(MC_ERR_INVALID, "render: too many pixels");
    if (p->spp < 0) return set_error(MC_ERR_INVALID, "render: spp must be >= 0");
    if (p->max_depth < 0 || p->max_depth > MC_MAX_DEPTH) return set_error(MC_ERR_INVALID, "render: max_depth must be in [0, %d]", MC_MAX_DEPTH);
    if (p->rng != MC_RNG_PHILOX && p->rng != MC_RNG_XORWOW) return set_error(MC_ERR_INVALID, "render: unknown rng mode");
    if (p->intersector != MC_ISECT_REFERENCE && p->intersector != MC_ISECT_WATERTIGHT) return set_error(MC_ERR_INVALID, "render: unknown intersector");
    if (p->queue_capacity < 0) return set_error(MC_ERR_INVALID, "render: queue_capacity must be >= 0");
    if (p->stack_entries < 0 || p->stack_entries > MC_STACK_CAPACITY)
        return set_error(MC_ERR_INVALID, "render: stack_entries must be in [0, %d]", MC_STACK_CAPACITY);
    if (p->trace_threads != 0 && p->trace_threads != 128 && p->trace_threads != 256)
        return set_error(MC_ERR_INVALID, "render: trace_threads must be 0, 128 or 256");
    if (p->env_sampling != MC_ENV_SAMPLE_CDF && p->env_sampling != MC_ENV_SAMPLE_ALIAS)
        return set_error(MC_ERR_INVALID, "render: unknown environment sampling mode");
    if (p->env_sampling == MC_ENV_SAMPLE_ALIAS && v->env.enabled && !env_alias_table(v->env))
        return set_error(MC_ERR_INVALID, "render: alias sampling needs an environment map made by mc_env_create");
    if (v->light_count > 0 && !v->lights) return set_error(MC_ERR_INVALID, "render: null light array");
    if (v->triangle_count > 0 && !v->tri_cold) return set_error(MC_ERR_INVALID, "render: null cold triangle array");
    return MC_OK;
}

static mc_status finish_stats(mc_context* ctx, const RenderTiming& tm, long long paths, mc_render_stats* stats) {
    int flags = 0;
    MC_CUDA(cudaMemcpyAsync(&flags, ctx->d_error, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        long long h[2 * MC_MAX_DEPTH_STATS + 8];
        MC_CUDA(cudaMemcpyAsync(h, ctx->d_stats, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
        MC_CUDA(cudaStreamSynchronize(ctx->stream));
        for (int d = 0; d < MC_MAX_DEPTH_STATS; d++) {
            stats->extend_per_depth[d] = h[d];
            stats->shadow_per_depth[d] = h[MC_MAX_DEPTH_STATS + d];
            stats->extend_rays += h[d];
            stats->shadow_rays += h[MC_MAX_DEPTH_STATS + d];
        }
        stats->node_visits = h[2 * MC_MAX_DEPTH_STATS];
        stats->leaf_tests = h[2 * MC_MAX_DEPTH_STATS + 1];
        stats->paths = paths;
        stats->render_ms = tm.ms;
        stats->trace_ms = tm.trace_ms;
        stats->shade_ms = tm.shade_ms;
        stats->guide_infer_ms = tm.infer_ms;
        stats->guide_train_ms = tm.train_ms;
        stats->trace_launches = tm.trace_launches;
        stats->kernel_launches = tm.kernel_launches;
        stats->error_flags = flags;
    } else {
        MC_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    return status_from_device_flags(flags);
}

mc_status render_items(mc_context* ctx, const mc_bvh* bvh, const WaveItem* items, int n, bool useGraph,
                       mc_render_stats* stats, mc_guide* guide, bool train) {
    MC_CUDA(cudaMemsetAsync(ctx->d_error, 0, sizeof(int), ctx->stream));
    MC_CUDA(cudaMemsetAsync(ctx->d_stats, 0, (2 * MC_MAX_DEPTH_STATS + 8) * sizeof(long long), ctx->stream));
    RenderTiming tm;
    mc_status st = run_waves(ctx, bvh, items, n, useGraph, stats != nullptr, &tm, guide, train);
    if (st != MC_OK) return st;
    long long paths = 0;
    for (int i = 0; i < n; i++) paths += (long long)items[i].p->width * items[i].p->height * items[i].p->spp;
    return finish_stats(ctx, tm, paths, stats);
}

// The single-scene trace arguments of the ray-set entry points.
static void ray_set_scene(TraceArgs& t, const mc_bvh* bvh, const mc_scene_view* scene) {
    set_single_scene(t, bvh, bvh->layout != MC_BVH_LAYOUT_BINARY ? bvh->wide_roots[0] : bvh->bin_roots[0], scene);
}

}  // namespace mc

namespace mc {
// Samples per pixel in one wave of a single-image render: the tail bounces
// (few rays, a few long traversals set the launch time) and the launch
// sequence are then paid once per wave.
int wave_samples(const mc_render_params* params) {
    const long long pixels = (long long)params->width * params->height;
    int k = 1;
    if (params->rng == MC_RNG_PHILOX && params->spp > 1) {
        if (params->samples_per_wave > 0) {
            k = std::min(params->samples_per_wave, params->spp);
        } else if (params->samples_per_wave == 0) {
            // up to 32M paths per wave (about 4.5 GB of path and queue state)
            const long long perWave = 32ll << 20;
            k = (int)std::max(1ll, std::min<long long>({perWave / std::max(pixels, 1ll), 16ll, (long long)params->spp}));
        }
    }
    if (params->queue_capacity > 0 && k > 1) k = 1;  // a fixed queue capacity is one image's paths
    if ((long long)k * pixels >= (1ll << 30)) k = 1;
    return k;
}
}  // namespace mc

extern "C" {

mc_status mc_rng_reset(mc_context* ctx, int32_t width, int32_t height, uint64_t seed) {
    if (!ctx || width <= 0 || height <= 0) return mc::set_error(MC_ERR_INVALID, "mc_rng_reset: bad argument");
    return mc::rng_reset(ctx, width * height, seed);
}

mc_status mc_render_wavefront(mc_context* ctx, const mc_bvh* bvh, const mc_scene_view* scene, const mc_render_params* params,
                              float* d_accum, mc_render_stats* stats) {
    if (!ctx || !bvh) return mc::set_error(MC_ERR_INVALID, "mc_render_wavefront: null argument");
    mc_status st = mc::check_params(params, scene);
    if (st != MC_OK) return st;
    if (!d_accum) return mc::set_error(MC_ERR_INVALID, "mc_render_wavefront: null accumulation buffer");
    if (bvh->nseg != 1) return mc::set_error(MC_ERR_INVALID, "mc_render_wavefront: a batch BVH renders with mc_render_batch");
    if (scene->sphere_count + scene->triangle_count != bvh->n) return mc::set_error(MC_ERR_INVALID, "render: the BVH was built for another scene");
    int pixels = params->width * params->height;
    if (params->rng == MC_RNG_XORWOW && (!ctx->rng_ready || ctx->rng_pixels < pixels || ctx->rng_seed != params->seed)) {
        if ((st = mc::rng_reset(ctx, pixels, params->seed)) != MC_OK) return st;
    }
    const int root = bvh->layout != MC_BVH_LAYOUT_BINARY ? bvh->wide_roots[0] : bvh->bin_roots[0];
    mc::WaveItem it{scene, params, d_accum, root, 0};
    it.spw = mc::wave_samples(params);
    return mc::render_items(ctx, bvh, &it, 1, params->use_graph != 0, stats);
}

mc_status mc_render_batch(mc_context* ctx, const mc_bvh* bvh, const mc_batch_item* items, int32_t count, int32_t use_graph,
                          mc_render_stats* stats) {
    if (!ctx || !bvh || !items || count < 1) return mc::set_error(MC_ERR_INVALID, "mc_render_batch: bad argument");
    if (count > MC_WAVE_MAX_SCENES) return mc::set_error(MC_ERR_INVALID, "mc_render_batch: at most %d scenes per batch", MC_WAVE_MAX_SCENES);
    if (count != bvh->nseg) return mc::set_error(MC_ERR_INVALID, "mc_render_batch: %d items for a BVH of %d scenes", count, bvh->nseg);
    std::vector<mc::WaveItem> its((size_t)count);
    long long capacity = 0;
    for (int i = 0; i < count; i++) {
        mc_status st = mc::check_params(&items[i].params, &items[i].scene);
        if (st != MC_OK) return st;
        if (!items[i].d_accum) return mc::set_error(MC_ERR_INVALID, "mc_render_batch: null accumulation buffer (item %d)", i);
        if (items[i].params.rng != MC_RNG_PHILOX) return mc::set_error(MC_ERR_INVALID, "mc_render_batch: batches use the counter-based RNG");
        int prims = items[i].scene.sphere_count + items[i].scene.triangle_count;
        int segPrims = (i + 1 < bvh->nseg ? bvh->seg_prim_off[i + 1] : bvh->n) - bvh->seg_prim_off[i];
        if (prims != segPrims) return mc::set_error(MC_ERR_INVALID, "mc_render_batch: item %d does not match scene %d of the BVH", i, i);
        capacity += (long long)items[i].params.width * items[i].params.height;
        its[i] = mc::WaveItem{&items[i].scene, &items[i].params, items[i].d_accum,
                              bvh->layout != MC_BVH_LAYOUT_BINARY ? bvh->wide_roots[i] : bvh->bin_roots[i], i};
    }
    if (capacity >= (1ll << 30)) return mc::set_error(MC_ERR_INVALID, "mc_render_batch: too many paths per wave");
    // samples per wave: an item's own setting, else balanced so that the
    // batch's paths fill W waves of about 32M paths each and every item ends
    // within those W waves: item i traces ceil(spp_i / W) samples per wave
    // (at least 1, at most 16). An item with many samples then shares every
    // wave instead of trailing alone through small waves after the others
    // finished; images do not depend on it (each pixel adds its samples in
    // sample order).
    long long totalPaths = 0;
    for (int i = 0; i < count; i++)
        totalPaths += (long long)items[i].params.width * items[i].params.height * std::max(1, items[i].params.spp);
    const long long waves = std::max(1ll, (totalPaths + (32ll << 20) - 1) / (32ll << 20));
    for (int i = 0; i < count; i++) {
        const int want = items[i].params.samples_per_wave;
        const long long balanced = std::max(1ll, std::min(16ll, (std::max(1, items[i].params.spp) + waves - 1) / waves));
        its[i].spw = want > 0 ? want : want == 0 ? (int)balanced : 1;
        if ((long long)items[i].params.width * items[i].params.height * its[i].spw >= (1ll << 30)) its[i].spw = 1;
    }
    return mc::render_items(ctx, bvh, its.data(), count, use_graph != 0, stats);
}

mc_status mc_render_guided(mc_context* ctx, const mc_bvh* bvh, const mc_scene_view* scene, const mc_render_params* params,
                           mc_guide* guide, int32_t train, float* d_accum, mc_render_stats* stats) {
    if (!ctx || !bvh || !guide) return mc::set_error(MC_ERR_INVALID, "mc_render_guided: null argument");
    mc_status st = mc::check_params(params, scene);
    if (st != MC_OK) return st;
    if (!d_accum) return mc::set_error(MC_ERR_INVALID, "mc_render_guided: null accumulation buffer");
    if (bvh->nseg != 1) return mc::set_error(MC_ERR_INVALID, "mc_render_guided: needs a single-scene BVH");
    if (scene->sphere_count + scene->triangle_count != bvh->n) return mc::set_error(MC_ERR_INVALID, "render: the BVH was built for another scene");
    if (params->rng != MC_RNG_PHILOX) return mc::set_error(MC_ERR_INVALID, "mc_render_guided: guided renders use the counter-based RNG");
    if (guide->ctx != ctx) return mc::set_error(MC_ERR_INVALID, "mc_render_guided: the guide belongs to another context");
    const int pixels = params->width * params->height;
    if (params->queue_capacity > 0 && params->queue_capacity < pixels)
        return mc::set_error(MC_ERR_INVALID, "mc_render_guided: queue capacity below width*height");
    // several samples per wave as for plain renders, but at most 4 by
    // default: the guide trains once per wave (with as many Adam steps per
    // sample as with one sample per wave), and every record of a wave comes
    // from the same weights, so shorter waves keep the feedback tighter
    int k = 1;
    if (params->spp > 1) {
        if (params->samples_per_wave > 0) k = std::min(params->samples_per_wave, params->spp);
        else if (params->samples_per_wave == 0)
            k = (int)std::max(1ll, std::min<long long>({(32ll << 20) / pixels, 4ll, (long long)params->spp}));
    }
    if (params->queue_capacity > 0) k = 1;
    if ((st = mc::guide_reserve_paths(guide, pixels * k)) != MC_OK) return st;
    mc::WaveItem it{scene, params, d_accum, bvh->layout != MC_BVH_LAYOUT_BINARY ? bvh->wide_roots[0] : bvh->bin_roots[0], 0};
    it.spw = k;
    return mc::render_items(ctx, bvh, &it, 1, false, stats, guide, train != 0);
}

mc_status mc_trace_closest(mc_context* ctx, const mc_bvh* bvh, const mc_scene_view* scene, const float* d_rays, int32_t n,
                           int32_t intersector, mc_packed_hit* d_hits) {
    if (!ctx || !bvh || !scene || !d_rays || !d_hits || n < 0) return mc::set_error(MC_ERR_INVALID, "mc_trace_closest: bad argument");
    const bool plain = (intersector & MC_TRACE_PLAIN) != 0;
    intersector &= ~MC_TRACE_PLAIN;
    if (intersector != MC_ISECT_REFERENCE && intersector != MC_ISECT_WATERTIGHT) return mc::set_error(MC_ERR_INVALID, "mc_trace_closest: unknown intersector");
    if (bvh->nseg != 1) return mc::set_error(MC_ERR_INVALID, "mc_trace_closest: needs a single-scene BVH");
    if (n == 0) return MC_OK;
    mc_status st;
    if ((st = mc::devbuf_reserve(ctx->scratch[5], 64)) != MC_OK) return st;
    int* work = (int*)ctx->scratch[5].ptr;
    MC_CUDA(cudaMemsetAsync(work, 0, sizeof(int), ctx->stream));
    MC_CUDA(cudaMemsetAsync(ctx->d_error, 0, sizeof(int), ctx->stream));
    mc::TraceArgs t;
    std::memset(&t, 0, sizeof(t));
    mc::ray_set_scene(t, bvh, scene);
    t.err = ctx->d_error;
    t.refill = 8;
    size_t N = (size_t)n;
    t.extN = n;
    t.ox = d_rays; t.oy = d_rays + N; t.oz = d_rays + 2 * N;
    t.dx = d_rays + 3 * N; t.dy = d_rays + 4 * N; t.dz = d_rays + 5 * N; t.time = d_rays + 6 * N;
    t.hits = d_hits;
    t.work = work;
    mc::launch_trace(ctx, ctx->stream, t, bvh->layout, false, intersector, !plain, (n + 255) / 256);
    MC_CUDA(cudaGetLastError());
    int flags = 0;
    MC_CUDA(cudaMemcpyAsync(&flags, ctx->d_error, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    MC_CUDA(cudaStreamSynchronize(ctx->stream));
    return mc::status_from_device_flags(flags);
}

mc_status mc_trace_any(mc_context* ctx, const mc_bvh* bvh, const mc_scene_view* scene, const float* d_rays, const float* d_tmax,
                       int32_t n, int32_t intersector, int32_t* d_occluded) {
    if (!ctx || !bvh || !scene || !d_rays || !d_tmax || !d_occluded || n < 0) return mc::set_error(MC_ERR_INVALID, "mc_trace_any: bad argument");
    const bool plain = (intersector & MC_TRACE_PLAIN) != 0;
    intersector &= ~MC_TRACE_PLAIN;
    if (intersector != MC_ISECT_REFERENCE && intersector != MC_ISECT_WATERTIGHT) return mc::set_error(MC_ERR_INVALID, "mc_trace_any: unknown intersector");
    if (bvh->nseg != 1) return mc::set_error(MC_ERR_INVALID, "mc_trace_any: needs a single-scene BVH");
    if (n == 0) return MC_OK;
    mc_status st;
    if ((st = mc::devbuf_reserve(ctx->scratch[5], 64)) != MC_OK) return st;
    int* work = (int*)ctx->scratch[5].ptr;
    MC_CUDA(cudaMemsetAsync(work, 0, sizeof(int), ctx->stream));
    MC_CUDA(cudaMemsetAsync(ctx->d_error, 0, sizeof(int), ctx->stream));
    mc::TraceArgs t;
    std::memset(&t, 0, sizeof(t));
    mc::ray_set_scene(t, bvh, scene);
    t.err = ctx->d_error;
    t.refill = 8;
    size_t N = (size_t)n;
    t.shN = n;
    t.sox = d_rays; t.soy = d_rays + N; t.soz = d_rays + 2 * N;
    t.sdx = d_rays + 3 * N; t.sdy = d_rays + 4 * N; t.sdz = d_rays + 5 * N;
    t.time = d_rays + 6 * N;
    t.smax = d_tmax;
    t.occluded = d_occluded;
    t.work = work;
    mc::launch_trace(ctx, ctx->stream, t, bvh->layout, false, intersector, !plain, (n + 255) / 256);
    MC_CUDA(cudaGetLastError());
    int flags = 0;
    MC_CUDA(cudaMemcpyAsync(&flags, ctx->d_error, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    MC_CUDA(cudaStreamSynchronize(ctx->stream));
    return mc::status_from_device_flags(flags);
}

}  // extern "C"
