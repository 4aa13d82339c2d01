// mc_traverse.cuh - BVH traversal over the library's node layout.
//
// Binary layout: one 64-byte record per internal node holding BOTH children's
// boxes and references (leaf child k -> ~k), so a traversal step is one
// contiguous 64-byte read instead of the reference's node read plus two child
// box reads (PT:1276-1321). Leaves are 48-byte primitive records in leaf
// (sorted Morton) order: a triangle's three vertices plus its id and type.
//
// The visit order and every test follow the reference's stepTraversal /
// traverseAnyHit (PT:1152-1321): both child boxes are tested against the
// current closest distance, a leaf child is intersected on the spot (left then
// right), internal children are descended left first with the right one
// pushed. Closest hits keep the first primitive found at equal t (strict <).
#pragma once
#include "mc_math.cuh"

// Leaf children of a 4-wide node: one loop over the lane's hit leaves (1) or
// one predicated block per child slot (0).
#ifndef MC_LEAF_LOOP
#define MC_LEAF_LOOP 1
#endif
// Traversal stack of the trace kernel: shared memory (1; 64 KB per 256-thread
// block, measured 2 % faster on B200) or local memory (0).
#ifndef MC_SMEM_STACK
#define MC_SMEM_STACK 1
#endif
// 4-wide steps: start fetching the next node (the nearest hit internal child,
// else the top of the stack) into L1 before the leaf children are intersected,
// so its latency overlaps theirs (1), or not (0).
#ifndef MC_PREFETCH_NEXT
#define MC_PREFETCH_NEXT 0
#endif

namespace mc {

enum { STEP_CONTINUE = 0, STEP_DONE = 1, STEP_OCCLUDED = 2 };

struct TraceScene {
    const float4* __restrict__ nodes;   // binary: 4 float4 per internal node; wide: 8
    const float4* __restrict__ prims;   // 3 float4 per leaf
    int root;                           // root node of this scene (batched builds share the arrays)
};

// A lane's traversal stack in local memory.
struct LocalStack {
    int* p;
    MC_D int& operator[](int i) const { return p[i]; }
};
// A lane's traversal stack in shared memory: entry i of the block's thread t at
// base[i * STRIDE + t], so a warp's accesses fall in 32 distinct banks at any depths.
template <int STRIDE>
struct SharedStack {
    int* p;  // base + threadIdx.x
    MC_D int& operator[](int i) const { return p[i * STRIDE]; }
};

// Traversal state of one ray in one lane.
struct TravState {
    RayInv r;
    float time;
    float tmax;     // closest distance so far (closest) or the segment length (any hit)
    int hitLeaf;    // leaf slot of the closest hit, -1 none
    int node;
    int sp;
};

MC_D void trav_begin(TravState& s, const V3& o, const V3& d, float time, float tmax, int root) {
    s.r = make_ray_inv(o, d);
    s.time = time;
    s.tmax = tmax;
    s.hitLeaf = -1;
    s.node = root;
    s.sp = 0;
}

MC_D float4 ldg4(const float4* p) { return __ldg(p); }

// Intersects leaf slot k; returns true and t when the primitive is hit with
// t in the reference's accepted range (hit_* internal checks).
template <int ISECT>
MC_D bool leaf_hit(const TraceScene& sc, int k, const TravState& s, const WatertightRay& w, float& t) {
    const float4* rec = sc.prims + (long long)k * 3;
    float4 a = ldg4(rec + 0), b = ldg4(rec + 1), c = ldg4(rec + 2);
    int type = __float_as_int(c.z);
    if (type == 1) {
        V3 v0(a.x, a.y, a.z), v1(a.w, b.x, b.y), v2(b.z, b.w, c.x);
        if (ISECT == 0) return hit_triangle_ref(v0, v1, v2, s.r.o, s.r.d, t);
        return hit_triangle_watertight(w, v0, v1, v2, s.r.o, t);
    }
    bool front;
    V3 outward;
    return hit_sphere_ref(V3(a.x, a.y, a.z), V3(a.w, b.x, b.y), b.w != 0.f, b.z, s.r.o, s.r.d, s.time, t, front, outward);
}

// One traversal step. ANY: any-hit semantics (PT:1152-1207): boxes are tested
// against the fixed segment length and the first blocker in (1e-4, tmax) ends
// the ray. Otherwise closest hit (PT:1276-1321 + testPrimitiveClosest 1537-1551).
// Counters of the instrumented variant: node visits and primitive tests.
struct TravCount {
    int visits = 0;
    int leaves = 0;
};

// cap: stack entries available to the lane (at most MC_STACK_CAPACITY); a push
// beyond it ends the ray and sets MC_DEVERR_STACK.
template <bool ANY, int ISECT, bool COUNT = false, class Stack = LocalStack>
MC_D int trav_step(const TraceScene& sc, TravState& s, const Stack& stack, const WatertightRay& w, int* err,
                   TravCount* cnt, int cap) {
    const float4* nd = sc.nodes + (long long)s.node * 4;
    float4 a = ldg4(nd + 0), b = ldg4(nd + 1), c = ldg4(nd + 2), d = ldg4(nd + 3);
    int lref = __float_as_int(d.x), rref = __float_as_int(d.y);
    bool oL = hit_box(s.r, a.x, a.y, a.z, a.w, b.x, b.y, s.tmax);
    bool oR = hit_box(s.r, b.z, b.w, c.x, c.y, c.z, c.w, s.tmax);
    bool lLeaf = lref < 0, rLeaf = rref < 0;
    if (COUNT) {
        cnt->visits++;
        cnt->leaves += (oL && lLeaf ? 1 : 0) + (oR && rLeaf ? 1 : 0);
    }
    if (oL && lLeaf) {
        float t;
        if (leaf_hit<ISECT>(sc, ~lref, s, w, t)) {
            if (ANY) {
                if (t > 0.0001f && t < s.tmax) return STEP_OCCLUDED;
            } else if (t < s.tmax && t > 0.0001f) {
                s.tmax = t;
                s.hitLeaf = ~lref;
            }
        }
    }
    if (oR && rLeaf) {
        float t;
        if (leaf_hit<ISECT>(sc, ~rref, s, w, t)) {
            if (ANY) {
                if (t > 0.0001f && t < s.tmax) return STEP_OCCLUDED;
            } else if (t < s.tmax && t > 0.0001f) {
                s.tmax = t;
                s.hitLeaf = ~rref;
            }
        }
    }
    bool tL = oL && !lLeaf, tR = oR && !rLeaf;
    if (!tL && !tR) {
        if (s.sp == 0) return STEP_DONE;
        s.sp--;
        s.node = stack[s.sp];
    } else {
        if (tL && tR) {
            if (s.sp >= cap) {
                atomicOr(err, MC_DEVERR_STACK);
                return STEP_DONE;
            }
            stack[s.sp] = rref;
            s.sp++;
        }
        s.node = tL ? lref : rref;
    }
    return STEP_CONTINUE;
}

// ---------------------------------------------------------------------------
// 4-wide layout: 128 bytes per node = child boxes as six float4 (lo.x, lo.y,
// lo.z, hi.x, hi.y, hi.z of the four children), the four child references
// (internal: wide-node index; leaf: ~rank; empty: MC_WIDE_EMPTY) and a spare
// float4. Leaves are stored in the reference's static visit order (their rank),
// so "first found at equal t" becomes "smallest rank at equal t" whatever order
// this traversal visits them in; every box is an exact box of the binary tree,
// tested with the reference's slab arithmetic (no per-axis early exit is needed:
// the three-axis test returns the same boolean).
// ---------------------------------------------------------------------------
MC_D void slab4(const RayInv& r, float lx, float ly, float lz, float hx, float hy, float hz, float tfar, float& tnear,
                bool& hit) {
    float e0 = (lx - r.o.x) * r.ix, x0 = (hx - r.o.x) * r.ix;
    if (r.ix < 0.0f) { float t = e0; e0 = x0; x0 = t; }
    float e1 = (ly - r.o.y) * r.iy, x1 = (hy - r.o.y) * r.iy;
    if (r.iy < 0.0f) { float t = e1; e1 = x1; x1 = t; }
    float e2 = (lz - r.o.z) * r.iz, x2 = (hz - r.o.z) * r.iz;
    if (r.iz < 0.0f) { float t = e2; e2 = x2; x2 = t; }
    float n = fmaxf(fmaxf(fmaxf(0.0001f, e0), e1), e2);
    float f = fminf(fminf(fminf(tfar, x0), x1), x2);
    hit = !(f <= n);
    tnear = n;
}

MC_D void cswap(float& ka, int& va, float& kb, int& vb) {
    if (kb < ka) {
        float tk = ka; ka = kb; kb = tk;
        int tv = va; va = vb; vb = tv;
    }
}

// Child planes of a quantised node (MC_BVH_LAYOUT_WIDE4Q): plane = origin +
// byte * 2^e, one byte per child in each word.
MC_D float4 q_planes(float origin, float scale, unsigned bytes) {
    return make_float4(fmaf((float)(bytes & 0xFFu), scale, origin), fmaf((float)((bytes >> 8) & 0xFFu), scale, origin),
                       fmaf((float)((bytes >> 16) & 0xFFu), scale, origin), fmaf((float)(bytes >> 24), scale, origin));
}

MC_D float q_scale(unsigned exps, int axis) {
    const int e = (int)((exps >> (8 * axis)) & 0xFFu) - 128;
    return __int_as_float((e + 127) << 23);
}

// QUANT: 64-byte quantised nodes with conservative boxes (more boxes pass; the
// leaf tests and the rank rule decide the hit as with exact boxes).
template <bool ANY, int ISECT, bool COUNT = false, class Stack = LocalStack, bool QUANT = false>
MC_D int trav_step4(const TraceScene& sc, TravState& s, const Stack& stack, const WatertightRay& w, int* err,
                    TravCount* cnt, int cap) {
    float4 lx, ly, lz, hx, hy, hz, rf;
    if (QUANT) {
        const float4* nd = sc.nodes + (long long)s.node * 4;
        const float4 h = ldg4(nd + 0), q0 = ldg4(nd + 1), q1 = ldg4(nd + 2);
        rf = ldg4(nd + 3);
        const unsigned ex = (unsigned)__float_as_int(h.w);
        const float sx = q_scale(ex, 0), sy = q_scale(ex, 1), sz = q_scale(ex, 2);
        lx = q_planes(h.x, sx, (unsigned)__float_as_int(q0.x));
        ly = q_planes(h.y, sy, (unsigned)__float_as_int(q0.y));
        lz = q_planes(h.z, sz, (unsigned)__float_as_int(q0.z));
        hx = q_planes(h.x, sx, (unsigned)__float_as_int(q0.w));
        hy = q_planes(h.y, sy, (unsigned)__float_as_int(q1.x));
        hz = q_planes(h.z, sz, (unsigned)__float_as_int(q1.y));
    } else {
        const float4* nd = sc.nodes + (long long)s.node * 8;
        lx = ldg4(nd + 0); ly = ldg4(nd + 1); lz = ldg4(nd + 2);
        hx = ldg4(nd + 3); hy = ldg4(nd + 4); hz = ldg4(nd + 5);
        rf = ldg4(nd + 6);
    }
    int ref[4] = {__float_as_int(rf.x), __float_as_int(rf.y), __float_as_int(rf.z), __float_as_int(rf.w)};
    float tn[4];
    bool hit[4];
    slab4(s.r, lx.x, ly.x, lz.x, hx.x, hy.x, hz.x, s.tmax, tn[0], hit[0]);
    slab4(s.r, lx.y, ly.y, lz.y, hx.y, hy.y, hz.y, s.tmax, tn[1], hit[1]);
    slab4(s.r, lx.z, ly.z, lz.z, hx.z, hy.z, hz.z, s.tmax, tn[2], hit[2]);
    slab4(s.r, lx.w, ly.w, lz.w, hx.w, hy.w, hz.w, s.tmax, tn[3], hit[3]);
    if (COUNT) cnt->visits++;
#if MC_PREFETCH_NEXT
    {
        // the next node does not depend on the leaf tests below: the hit flags
        // are taken against the distance before them, as in the choice further down
        float kn = INFINITY;
        int vn = -1;
#pragma unroll
        for (int c = 0; c < 4; c++)
            if (hit[c] && ref[c] >= 0 && ref[c] != MC_WIDE_EMPTY && tn[c] < kn) {
                kn = tn[c];
                vn = ref[c];
            }
        if (vn < 0 && s.sp > 0) vn = stack[s.sp - 1];
        if (vn >= 0) {
            const float4* nn = sc.nodes + (long long)vn * (QUANT ? 4 : 8);
            asm volatile("prefetch.global.L1 [%0];" ::"l"(nn));
        }
    }
#endif
    // leaf children first
#if MC_LEAF_LOOP
    // one loop over this lane's hit leaf children: a warp runs as many
    // iterations as its busiest lane, not one predicated block per child slot
    unsigned lm = (hit[0] && ref[0] < 0 ? 1u : 0u) | (hit[1] && ref[1] < 0 ? 2u : 0u) |
                  (hit[2] && ref[2] < 0 ? 4u : 0u) | (hit[3] && ref[3] < 0 ? 8u : 0u);
    while (lm) {
        const int c = __ffs(lm) - 1;
        lm &= lm - 1;
        const int k = ~(c == 0 ? ref[0] : c == 1 ? ref[1] : c == 2 ? ref[2] : ref[3]);
        float t;
        if (COUNT) cnt->leaves++;
        if (leaf_hit<ISECT>(sc, k, s, w, t)) {
            if (ANY) {
                if (t > 0.0001f && t < s.tmax) return STEP_OCCLUDED;
            } else if (t > 0.0001f && (t < s.tmax || (t == s.tmax && s.hitLeaf >= 0 && k < s.hitLeaf))) {
                s.tmax = t;
                s.hitLeaf = k;
            }
        }
    }
#else
#pragma unroll
    for (int c = 0; c < 4; c++) {
        if (hit[c] && ref[c] < 0) {
            int k = ~ref[c];
            float t;
            if (COUNT) cnt->leaves++;
            if (leaf_hit<ISECT>(sc, k, s, w, t)) {
                if (ANY) {
                    if (t > 0.0001f && t < s.tmax) return STEP_OCCLUDED;
                } else if (t > 0.0001f && (t < s.tmax || (t == s.tmax && s.hitLeaf >= 0 && k < s.hitLeaf))) {
                    s.tmax = t;
                    s.hitLeaf = k;
                }
            }
        }
    }
#endif
    // internal children, nearest first: sort (tnear, ref) ascending, misses as +inf
    float k0 = (hit[0] && ref[0] >= 0 && ref[0] != MC_WIDE_EMPTY) ? tn[0] : INFINITY;
    float k1 = (hit[1] && ref[1] >= 0 && ref[1] != MC_WIDE_EMPTY) ? tn[1] : INFINITY;
    float k2 = (hit[2] && ref[2] >= 0 && ref[2] != MC_WIDE_EMPTY) ? tn[2] : INFINITY;
    float k3 = (hit[3] && ref[3] >= 0 && ref[3] != MC_WIDE_EMPTY) ? tn[3] : INFINITY;
    int v0 = ref[0], v1 = ref[1], v2 = ref[2], v3 = ref[3];
    cswap(k0, v0, k1, v1);
    cswap(k2, v2, k3, v3);
    cswap(k0, v0, k2, v2);
    cswap(k1, v1, k3, v3);
    cswap(k1, v1, k2, v2);
    if (k0 == INFINITY) {
        if (s.sp == 0) return STEP_DONE;
        s.sp--;
        s.node = stack[s.sp];
        return STEP_CONTINUE;
    }
    // push the farther ones (farthest first), continue with the nearest
    int extra = (k1 != INFINITY) + (k2 != INFINITY) + (k3 != INFINITY);
    if (s.sp + extra > cap) {
        atomicOr(err, MC_DEVERR_STACK);
        return STEP_DONE;
    }
    if (k3 != INFINITY) stack[s.sp++] = v3;
    if (k2 != INFINITY) stack[s.sp++] = v2;
    if (k1 != INFINITY) stack[s.sp++] = v1;
    s.node = v0;
    return STEP_CONTINUE;
}

// LAY: MC_BVH_LAYOUT_BINARY, _WIDE4 or _WIDE4Q.
template <bool ANY, int ISECT, bool COUNT, int LAY, class Stack>
MC_D int trav_step_layout(const TraceScene& sc, TravState& s, const Stack& stack, const WatertightRay& w, int* err,
                          TravCount* cnt, int cap) {
    if (LAY == MC_BVH_LAYOUT_WIDE4Q) return trav_step4<ANY, ISECT, COUNT, Stack, true>(sc, s, stack, w, err, cnt, cap);
    if (LAY == MC_BVH_LAYOUT_WIDE4) return trav_step4<ANY, ISECT, COUNT, Stack, false>(sc, s, stack, w, err, cnt, cap);
    return trav_step<ANY, ISECT, COUNT, Stack>(sc, s, stack, w, err, cnt, cap);
}

// The hit record fields a leaf slot stands for.
MC_D void leaf_identity(const TraceScene& sc, int k, int& type, int& id) {
    float4 c = ldg4(sc.prims + (long long)k * 3 + 2);
    id = __float_as_int(c.y);
    type = __float_as_int(c.z);
}

}  // namespace mc
