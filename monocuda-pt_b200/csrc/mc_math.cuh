// mc_math.cuh - vector arithmetic and the reference's per-ray math, restated.
//
// Parity with the reference depends on evaluating every expression in the same
// algebraic form the reference uses (same operand order, same divisions, same
// places where nvcc may contract a multiply-add), because the reference is
// built with --use_fast_math (CMakeLists.txt:94-96) and so is the render code
// here. Each function cites the reference function whose steps it follows
// (path_tracer.cu, "PT" below).
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#define MC_HD __host__ __device__ __forceinline__
#define MC_D __device__ __forceinline__
#define MC_PI 3.14159265358979323846f

namespace mc {

// PT:105-158 vec3. Member-wise operators; normalize divides each component.
struct V3 {
    float x, y, z;
    MC_HD V3() : x(0), y(0), z(0) {}
    MC_HD V3(float a, float b, float c) : x(a), y(b), z(c) {}
    MC_HD V3 operator+(const V3& o) const { return V3{x + o.x, y + o.y, z + o.z}; }
    MC_HD V3 operator-(const V3& o) const { return V3{x - o.x, y - o.y, z - o.z}; }
    MC_HD V3 operator*(const V3& o) const { return V3{x * o.x, y * o.y, z * o.z}; }
    MC_HD V3 operator-() const { return V3{-x, -y, -z}; }
    MC_HD V3 operator*(float s) const { return V3{x * s, y * s, z * s}; }
    MC_HD V3 operator/(float s) const { return V3{x / s, y / s, z / s}; }
    MC_HD float length_squared() const { return x * x + y * y + z * z; }
    MC_HD float length() const { return sqrtf(length_squared()); }
    MC_HD V3 cross(const V3& o) const { return {y * o.z - z * o.y, z * o.x - x * o.z, x * o.y - y * o.x}; }
    MC_HD float dot(const V3& o) const { return x * o.x + y * o.y + z * o.z; }
    MC_HD V3 normalize() const {
        float len = sqrtf(length_squared());
        return V3{x / len, y / len, z / len};
    }
    MC_HD V3 reflect(const V3& n) const { return *this - n * (2.0f * dot(n)); }
};

struct V2 {
    float x, y;
    MC_HD V2() : x(0), y(0) {}
    MC_HD V2(float a, float b) : x(a), y(b) {}
    MC_HD V2 operator+(const V2& o) const { return V2{x + o.x, y + o.y}; }
    MC_HD V2 operator*(float s) const { return V2{x * s, y * s}; }
};

// PT:141-156 vec3::refract
MC_D V3 refract(const V3& self, const V3& n, float eta) {
    V3 direction = self.normalize();
    float cosTheta1 = fminf((-direction).dot(n), 1.0f);
    float theta1 = acosf(cosTheta1);
    float sinTheta2 = sinf(theta1) * eta;
    if (sinTheta2 > 1.f) return direction.reflect(n);
    float theta2 = asinf(sinTheta2);
    V3 tangent = direction + n * cosTheta1;
    float tangentLength = tangent.length();
    if (tangentLength > 1e-8f) tangent = tangent / tangentLength;
    return tangent * sinf(theta2) - n * cosf(theta2);
}

// ---------------------------------------------------------------------------
// Ray / box. PT:1467-1488 hit_aabb computes 1/d per axis per box; the inverse
// here is computed once per ray (rcp is deterministic, so the value is the same)
// and the per-axis steps are unrolled in the reference's x, y, z order.
// ---------------------------------------------------------------------------
struct RayInv {
    V3 o, d;
    float ix, iy, iz;
};

MC_D RayInv make_ray_inv(const V3& o, const V3& d) {
    RayInv r;
    r.o = o;
    r.d = d;
    r.ix = 1.0f / d.x;
    r.iy = 1.0f / d.y;
    r.iz = 1.0f / d.z;
    return r;
}

MC_D bool slab_axis(float lo, float hi, float o, float inv, float& tnear, float& tfar) {
    float entry = (lo - o) * inv;
    float exit = (hi - o) * inv;
    if (inv < 0.0f) {
        float t = entry;
        entry = exit;
        exit = t;
    }
    tnear = fmaxf(tnear, entry);
    tfar = fminf(tfar, exit);
    return !(tfar <= tnear);
}

// near starts at 1e-4, far at the current closest distance (PT:1107-1113).
MC_D bool hit_box(const RayInv& r, float lox, float loy, float loz, float hix, float hiy, float hiz, float tfar) {
    float tnear = 0.0001f;
    if (!slab_axis(lox, hix, r.o.x, r.ix, tnear, tfar)) return false;
    if (!slab_axis(loy, hiy, r.o.y, r.iy, tnear, tfar)) return false;
    if (!slab_axis(loz, hiz, r.o.z, r.iz, tnear, tfar)) return false;
    return true;
}

// ---------------------------------------------------------------------------
// Ray / triangle, PT:715-741 hit_triangle (plane + three edge signs; the
// reference's test, not watertight).
// ---------------------------------------------------------------------------
MC_D bool hit_triangle_ref(const V3& v0, const V3& v1, const V3& v2, const V3& o, const V3& d, float& tout) {
    V3 edge1 = v1 - v0;
    V3 edge2 = v2 - v0;
    V3 nrm = edge1.cross(edge2).normalize();
    float denom = d.dot(nrm);
    if (fabsf(denom) < 1e-6f) return false;
    float t = (v0 - o).dot(nrm) / denom;
    if (t < 0.0001f) return false;
    V3 p = o + d * t;
    V3 e0 = v1 - v0;
    V3 p0 = p - v0;
    if (nrm.dot(e0.cross(p0)) < 0) return false;
    V3 e1 = v2 - v1;
    V3 p1 = p - v1;
    if (nrm.dot(e1.cross(p1)) < 0) return false;
    V3 e2 = v0 - v2;
    V3 p2 = p - v2;
    if (nrm.dot(e2.cross(p2)) < 0) return false;
    tout = t;
    return true;
}

// Watertight ray/triangle test (Woop, Benthin, Wald, "Watertight Ray/Triangle
// Intersection", JCGT 2013): shear/scale into ray space, edge functions with a
// double-precision fallback on exact zeros, no epsilon on the edges.
struct WatertightRay {
    int kx, ky, kz;
    float sx, sy, sz;
};

MC_D WatertightRay make_watertight(const V3& d) {
    WatertightRay w;
    float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    int kz = (ax > ay) ? ((ax > az) ? 0 : 2) : ((ay > az) ? 1 : 2);
    int kx = kz + 1; if (kx == 3) kx = 0;
    int ky = kx + 1; if (ky == 3) ky = 0;
    float dk[3] = {d.x, d.y, d.z};
    if (dk[kz] < 0.0f) { int t = kx; kx = ky; ky = t; }
    w.kx = kx; w.ky = ky; w.kz = kz;
    w.sx = __fdiv_rn(dk[kx], dk[kz]);
    w.sy = __fdiv_rn(dk[ky], dk[kz]);
    w.sz = __fdiv_rn(1.0f, dk[kz]);
    return w;
}

MC_D float comp(const V3& v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

MC_D bool hit_triangle_watertight(const WatertightRay& w, const V3& v0, const V3& v1, const V3& v2, const V3& o,
                                  float& tout) {
    V3 a = v0 - o, b = v1 - o, c = v2 - o;
    float ax = __fsub_rn(comp(a, w.kx), __fmul_rn(w.sx, comp(a, w.kz)));
    float ay = __fsub_rn(comp(a, w.ky), __fmul_rn(w.sy, comp(a, w.kz)));
    float bx = __fsub_rn(comp(b, w.kx), __fmul_rn(w.sx, comp(b, w.kz)));
    float by = __fsub_rn(comp(b, w.ky), __fmul_rn(w.sy, comp(b, w.kz)));
    float cx = __fsub_rn(comp(c, w.kx), __fmul_rn(w.sx, comp(c, w.kz)));
    float cy = __fsub_rn(comp(c, w.ky), __fmul_rn(w.sy, comp(c, w.kz)));
    float U = __fsub_rn(__fmul_rn(cx, by), __fmul_rn(cy, bx));
    float V = __fsub_rn(__fmul_rn(ax, cy), __fmul_rn(ay, cx));
    float W = __fsub_rn(__fmul_rn(bx, ay), __fmul_rn(by, ax));
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        double CxBy = (double)cx * (double)by, CyBx = (double)cy * (double)bx;
        U = (float)(CxBy - CyBx);
        double AxCy = (double)ax * (double)cy, AyCx = (double)ay * (double)cx;
        V = (float)(AxCy - AyCx);
        double BxAy = (double)bx * (double)ay, ByAx = (double)by * (double)ax;
        W = (float)(BxAy - ByAx);
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    float det = __fadd_rn(__fadd_rn(U, V), W);
    if (det == 0.0f) return false;
    float az = __fmul_rn(w.sz, comp(a, w.kz));
    float bz = __fmul_rn(w.sz, comp(b, w.kz));
    float cz = __fmul_rn(w.sz, comp(c, w.kz));
    float T = __fadd_rn(__fadd_rn(__fmul_rn(U, az), __fmul_rn(V, bz)), __fmul_rn(W, cz));
    float t = __fdiv_rn(T, det);
    if (!(t >= 0.0001f)) return false;
    tout = t;
    return true;
}

// ---------------------------------------------------------------------------
// Ray / sphere, PT:886-911 hit_sphere (center_at PT:871-873).
// ---------------------------------------------------------------------------
MC_D V3 sphere_center_at(const V3& c0, const V3& c1, bool moving, float time) {
    return moving ? c0 + (c1 - c0) * time : c0;
}

MC_D bool hit_sphere_ref(const V3& c0, const V3& c1, bool moving, float radius, const V3& o, const V3& d, float time,
                         float& tout, bool& frontFace, V3& outward) {
    V3 cc = sphere_center_at(c0, c1, moving, time);
    V3 oc = cc - o;
    float tc = oc.dot(d) / d.dot(d);
    V3 closest = o + d * tc;
    float dist2 = (cc - closest).length_squared();
    float disc = radius * radius - dist2;
    if (disc < 0.0f) return false;
    float half = sqrtf(disc);
    float nearRoot = tc - half;
    float farRoot = tc + half;
    float t = nearRoot;
    if (t < 0.0001f) t = farRoot;
    if (t < 0.0001f) return false;
    V3 p = o + d * t;
    outward = (p - cc).normalize();
    frontFace = d.dot(outward) < 0.0f;
    tout = t;
    return true;
}

// PT:862-869 computeSphereUvFromOutwardNormal
MC_D V2 sphere_uv(const V3& n) {
    float clampedNegativeY = fminf(1.0f, fmaxf(-1.0f, -n.y));
    float theta = acosf(clampedNegativeY);
    float phi = atan2f(-n.z, n.x) + MC_PI;
    return V2(phi / (2.0f * MC_PI), theta / MC_PI);
}

// PT:687-695 computeTriangleUvFromHitPoint
MC_D V2 triangle_uv(const V3& v0, const V3& v1, const V3& v2, const V2& uv0, const V2& uv1, const V2& uv2, const V3& p) {
    float area2 = (v1 - v0).cross(v2 - v0).length();
    float w0 = (v1 - p).cross(v2 - p).length() / area2;
    float w1 = (v0 - p).cross(v2 - p).length() / area2;
    float w2 = (v1 - p).cross(v0 - p).length() / area2;
    return uv0 * w0 + uv1 * w1 + uv2 * w2;
}

// PT:697-713 computeTriangleShadingNormal
MC_D V3 triangle_shading_normal(const V3& v0, const V3& v1, const V3& v2, const V3& n0, const V3& n1, const V3& n2,
                                const V3& p, const V3& faceNormal) {
    if (n0.length_squared() == 0.0f) return faceNormal;
    float area2 = (v1 - v0).cross(v2 - v0).length();
    float w0 = (v1 - p).cross(v2 - p).length() / area2;
    float w1 = (v0 - p).cross(v2 - p).length() / area2;
    float w2 = (v1 - p).cross(v0 - p).length() / area2;
    float ws = w0 + w1 + w2;
    if (!(ws > 0.0f) || ws > 1.01f) return faceNormal;
    V3 s = n0 * w0 + n1 * w1 + n2 * w2;
    if (s.length_squared() < 1e-12f) return faceNormal;
    s = s.normalize();
    if (s.dot(faceNormal) < 0.0f) s = -s;
    return s;
}

// PT:757-761, 763-765, 768-780, 837-843
MC_D float power_heuristic(float a, float b) {
    float a2 = a * a;
    float b2 = b * b;
    return a2 / (a2 + b2);
}
MC_D float lambertian_cosine_pdf(float c) { return c / MC_PI; }
MC_D float hg_phase_pdf(float cosTheta, float g) {
    float g2 = g * g;
    float denom = fmaxf(1.0f + g2 - 2.0f * g * cosTheta, 1e-6f);
    return (1.0f - g2) / (4.0f * MC_PI * denom * sqrtf(denom));
}
MC_D float triangle_area(const V3& v0, const V3& v1, const V3& v2) { return 0.5f * (v1 - v0).cross(v2 - v0).length(); }
MC_D float light_solid_angle_pdf(float sel, float dist, float cosL, float area) {
    return sel * (dist * dist) / (cosL * area);
}

// PT:476-480
MC_D float schlick(float cosine, float eta) {
    float r0 = (1.f - eta) / (1.f + eta);
    r0 = r0 * r0;
    return r0 + (1.f - r0) * powf((1 - cosine), 5.f);
}

}  // namespace mc
