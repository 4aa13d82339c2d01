// mc_oracle.cpp - CPU restatement of the reference's render hot path.
//
// TEST INFRASTRUCTURE (see mc_oracle.h). Compiled with g++ -ffp-contract=off,
// IEEE arithmetic. Every function cites the reference function
// (path_tracer.cu, "PT") whose steps it restates. Floating-point results are
// templated on the scalar type: float mirrors the reference's single precision
// on the CPU (no fast-math approximations), double is the FP64 estimator.
#include "mc_oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

namespace {

constexpr double kPiD = 3.14159265358979323846;

template <class T>
struct V {
    T x, y, z;
    V() : x(0), y(0), z(0) {}
    V(T a, T b, T c) : x(a), y(b), z(c) {}
    V operator+(const V& o) const { return V(x + o.x, y + o.y, z + o.z); }
    V operator-(const V& o) const { return V(x - o.x, y - o.y, z - o.z); }
    V operator*(const V& o) const { return V(x * o.x, y * o.y, z * o.z); }
    V operator-() const { return V(-x, -y, -z); }
    V operator*(T s) const { return V(x * s, y * s, z * s); }
    V operator/(T s) const { return V(x / s, y / s, z / s); }
    T len2() const { return x * x + y * y + z * z; }
    T len() const { return std::sqrt(len2()); }
    V cross(const V& o) const { return V(y * o.z - z * o.y, z * o.x - x * o.z, x * o.y - y * o.x); }
    T dot(const V& o) const { return x * o.x + y * o.y + z * o.z; }
    V norm() const {
        T l = std::sqrt(len2());
        return V(x / l, y / l, z / l);
    }
    V reflect(const V& n) const { return *this - n * (T(2) * dot(n)); }
};

template <class T>
V<T> vin(const mc_vec3& v) { return V<T>((T)v.x, (T)v.y, (T)v.z); }

// ---------------------------------------------------------------------------
// Philox-4x32-10 (Salmon et al. SC'11) and the draw mapping shared with the
// library's counter-based mode.
// ---------------------------------------------------------------------------
void philox(uint32_t c[4], uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; r++) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c[0], p1 = (uint64_t)0xCD9E8D57u * c[2];
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
        c[0] = n0; c[1] = (uint32_t)p1; c[2] = n2; c[3] = (uint32_t)p0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

struct Rng {
    uint32_t k0, k1, sample, pixel, draw;
    float uniform() {
        uint32_t c[4] = {draw >> 2, sample, pixel, 0u};
        philox(c, k0, k1);
        uint32_t w = c[draw & 3u];
        draw++;
        return ((float)(w >> 9) + 0.5f) * 1.1920928955078125e-07f;
    }
};

// ---------------------------------------------------------------------------
// Build (PT:913-935, 1337-1465, 1930-1987).
// ---------------------------------------------------------------------------
struct Box {
    float lx, ly, lz, hx, hy, hz;
};
Box merge(const Box& a, const Box& b) {
    return Box{std::fmin(a.lx, b.lx), std::fmin(a.ly, b.ly), std::fmin(a.lz, b.lz),
               std::fmax(a.hx, b.hx), std::fmax(a.hy, b.hy), std::fmax(a.hz, b.hz)};
}
mc_aabb to_aabb(const Box& b) {
    mc_aabb a;
    a.lo = mc_vec3{b.lx, b.ly, b.lz};
    a.hi = mc_vec3{b.hx, b.hy, b.hz};
    a.pad0 = a.pad1 = 0.f;
    return a;
}
Box from_aabb(const mc_aabb& a) { return Box{a.lo.x, a.lo.y, a.lo.z, a.hi.x, a.hi.y, a.hi.z}; }

uint32_t expand_bits(uint32_t p) {
    uint32_t e = 0;
    for (int i = 0; i < 10; i++) e |= ((p >> i) & 1u) << (3 * i);
    return e;
}
uint32_t quantize(float v, float lo, float hi) {
    float n = (v - lo) / (hi - lo);
    float s = n * 1023.0f;
    if (s != s) return 0u;
    return (uint32_t)(long long)s;
}

void prim_box(const mc_triangle* tris, const mc_sphere* sph, int ns, int i, Box& b, float c[3]) {
    if (i < ns) {
        const mc_sphere& s = sph[i];
        float r = s.radius;
        Box b0{s.center.x - r, s.center.y - r, s.center.z - r, s.center.x + r, s.center.y + r, s.center.z + r};
        if (s.is_moving) {
            Box b1{s.center1.x - r, s.center1.y - r, s.center1.z - r, s.center1.x + r, s.center1.y + r, s.center1.z + r};
            b = merge(b0, b1);
            c[0] = (s.center.x + s.center1.x) * 0.5f;
            c[1] = (s.center.y + s.center1.y) * 0.5f;
            c[2] = (s.center.z + s.center1.z) * 0.5f;
        } else {
            b = b0;
            c[0] = s.center.x; c[1] = s.center.y; c[2] = s.center.z;
        }
    } else {
        const mc_triangle& t = tris[i - ns];
        const float e = 1e-3f;
        b.lx = std::fmin(t.v0.x, std::fmin(t.v1.x, t.v2.x)) - e;
        b.ly = std::fmin(t.v0.y, std::fmin(t.v1.y, t.v2.y)) - e;
        b.lz = std::fmin(t.v0.z, std::fmin(t.v1.z, t.v2.z)) - e;
        b.hx = std::fmax(t.v0.x, std::fmax(t.v1.x, t.v2.x)) + e;
        b.hy = std::fmax(t.v0.y, std::fmax(t.v1.y, t.v2.y)) + e;
        b.hz = std::fmax(t.v0.z, std::fmax(t.v1.z, t.v2.z)) + e;
        c[0] = (t.v0.x + t.v1.x + t.v2.x) / 3.0f;
        c[1] = (t.v0.y + t.v1.y + t.v2.y) / 3.0f;
        c[2] = (t.v0.z + t.v1.z + t.v2.z) / 3.0f;
    }
}

int clz32(uint32_t v) { return v ? __builtin_clz(v) : 32; }
int delta(const uint32_t* codes, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    if (codes[i] == codes[j]) return 32 + clz32((uint32_t)(i ^ j));
    return clz32(codes[i] ^ codes[j]);
}

void karras(const uint32_t* codes, int n, int idx, int& left, int& right, bool& lLeaf, bool& rLeaf) {
    int d = (delta(codes, n, idx, idx + 1) - delta(codes, n, idx, idx - 1)) >= 0 ? 1 : -1;
    int dmin = delta(codes, n, idx, idx - d);
    int lmax = 2;
    while (delta(codes, n, idx, idx + lmax * d) > dmin) lmax *= 2;
    int l = 0;
    for (int t = lmax / 2; t >= 1; t /= 2)
        if (delta(codes, n, idx, idx + (l + t) * d) > dmin) l += t;
    int j = idx + l * d;
    int first = std::min(idx, j), last = std::max(idx, j);
    int common = delta(codes, n, first, last);
    int split = first, step = last - first;
    do {
        step = (step + 1) >> 1;
        int ns = split + step;
        if (ns < last && delta(codes, n, first, ns) > common) split = ns;
    } while (step > 1);
    left = split;
    right = split + 1;
    lLeaf = split == first;
    rLeaf = split + 1 == last;
}

// ---------------------------------------------------------------------------
// Intersection (PT:715-741, 886-911, 1467-1488) in precision T.
// ---------------------------------------------------------------------------
template <class T>
bool hit_aabb(const Box& b, const V<T>& o, const V<T>& d, T near, T far) {
    const T lo[3] = {(T)b.lx, (T)b.ly, (T)b.lz}, hi[3] = {(T)b.hx, (T)b.hy, (T)b.hz};
    const T oo[3] = {o.x, o.y, o.z}, dd[3] = {d.x, d.y, d.z};
    for (int a = 0; a < 3; a++) {
        T inv = T(1) / dd[a];
        T e = (lo[a] - oo[a]) * inv, x = (hi[a] - oo[a]) * inv;
        if (inv < T(0)) std::swap(e, x);
        near = std::fmax(near, e);
        far = std::fmin(far, x);
        if (far <= near) return false;
    }
    return true;
}

template <class T>
bool hit_triangle(const V<T>& v0, const V<T>& v1, const V<T>& v2, const V<T>& o, const V<T>& d, T& tout) {
    V<T> e1 = v1 - v0, e2 = v2 - v0;
    V<T> n = e1.cross(e2).norm();
    T den = d.dot(n);
    if (std::fabs(den) < T(1e-6f)) return false;
    T t = (v0 - o).dot(n) / den;
    if (t < T(0.0001f)) return false;
    V<T> p = o + d * t;
    if (n.dot((v1 - v0).cross(p - v0)) < 0) return false;
    if (n.dot((v2 - v1).cross(p - v1)) < 0) return false;
    if (n.dot((v0 - v2).cross(p - v2)) < 0) return false;
    tout = t;
    return true;
}

template <class T>
bool hit_sphere(const mc_sphere& s, const V<T>& o, const V<T>& d, T time, T& tout, bool& front, V<T>& outward) {
    V<T> c0 = vin<T>(s.center), c1 = vin<T>(s.center1);
    V<T> c = s.is_moving ? c0 + (c1 - c0) * time : c0;
    V<T> oc = c - o;
    T tc = oc.dot(d) / d.dot(d);
    V<T> cp = o + d * tc;
    T disc = (T)s.radius * (T)s.radius - (c - cp).len2();
    if (disc < T(0)) return false;
    T h = std::sqrt(disc);
    T t = tc - h;
    if (t < T(0.0001f)) t = tc + h;
    if (t < T(0.0001f)) return false;
    V<T> p = o + d * t;
    outward = (p - c).norm();
    front = d.dot(outward) < T(0);
    tout = t;
    return true;
}

struct Bvh {
    int n = 0;
    std::vector<mc_bvh_node> internal, leaves;
    std::vector<int32_t> types;
};

// closest (mode 0) or any (mode 1) over the reference's visit order
template <class T>
int traverse(const Bvh& b, const mc_triangle_hot* hot, const mc_sphere* sph, const V<T>& o, const V<T>& d, T time, T tmax,
             bool any, T& tout, bool& occluded) {
    int stack[128];
    int sp = 0, node = 0;
    T closest = tmax;
    int hitPrim = -1, hitType = -1;
    occluded = false;
    auto test = [&](int leaf) -> bool {
        int prim = b.leaves[leaf].prim, type = b.types[leaf];
        T t;
        bool ok;
        if (type == 0) {
            bool f;
            V<T> ow;
            ok = hit_sphere<T>(sph[prim], o, d, time, t, f, ow);
        } else {
            const mc_triangle_hot& h = hot[prim];
            ok = hit_triangle<T>(vin<T>(h.v0), vin<T>(h.v1), vin<T>(h.v2), o, d, t);
        }
        if (!ok) return false;
        if (any) return t > T(0.0001f) && t < tmax;
        if (t < closest && t > T(0.0001f)) {
            closest = t;
            hitPrim = prim;
            hitType = type;
        }
        return false;
    };
    if (b.n == 1) {
        if (hit_aabb<T>(from_aabb(b.leaves[0].bounds), o, d, T(0.0001f), closest)) occluded = test(0);
    } else {
        while (true) {
            const mc_bvh_node& nd = b.internal[node];
            const mc_aabb& lb = nd.left_is_leaf ? b.leaves[nd.left].bounds : b.internal[nd.left].bounds;
            const mc_aabb& rb = nd.right_is_leaf ? b.leaves[nd.right].bounds : b.internal[nd.right].bounds;
            T far = any ? tmax : closest;
            bool oL = hit_aabb<T>(from_aabb(lb), o, d, T(0.0001f), far);
            bool oR = hit_aabb<T>(from_aabb(rb), o, d, T(0.0001f), far);
            if (oL && nd.left_is_leaf && test(nd.left)) { occluded = true; break; }
            if (oR && nd.right_is_leaf && test(nd.right)) { occluded = true; break; }
            bool tL = oL && !nd.left_is_leaf, tR = oR && !nd.right_is_leaf;
            if (!tL && !tR) {
                if (sp == 0) break;
                node = stack[--sp];
            } else {
                if (tL && tR) {
                    if (sp >= 128) break;
                    stack[sp++] = nd.right;
                }
                node = tL ? nd.left : nd.right;
            }
        }
    }
    tout = closest;
    return hitPrim < 0 ? -1 : ((hitType << 30) | hitPrim);
}

void build_bvh(const mc_triangle* tris, int nt, const mc_sphere* sph, int ns, Bvh& out, std::vector<mc_aabb>* boxesOut = nullptr) {
    int n = nt + ns;
    std::vector<uint32_t> codes(n), sorted(n);
    std::vector<int32_t> perm(n);
    std::vector<mc_aabb> boxes(n);
    mc_aabb sb;
    orc_finalize_sort(tris, nt, sph, ns, codes.data(), sorted.data(), perm.data(), boxes.data(), &sb);
    out.n = n;
    out.internal.assign(std::max(1, n - 1), mc_bvh_node());
    out.leaves.assign(n, mc_bvh_node());
    orc_build(sorted.data(), perm.data(), boxes.data(), n, ns, out.internal.data(), out.leaves.data());
    out.types.resize(n);
    for (int k = 0; k < n; k++) out.types[k] = perm[k] < ns ? 0 : 1;
    if (boxesOut) *boxesOut = boxes;
}

// ---------------------------------------------------------------------------
// Environment map (PT:322-467) with the texture unit's bilinear filter
// restated (CUDA Programming Guide, texture fetching: weights in 9-bit fixed
// point with 8 fractional bits; wrap in u, clamp in v).
// ---------------------------------------------------------------------------
struct Env {
    bool enabled = false;
    int W = 0, H = 0;
    float intensity = 1.f, rotation = 0.f, total = 0.f;
    std::vector<float> rgba, rowCdf, colCdf;
};

void env_tables(Env& e) {
    e.rowCdf.assign(e.H + 1, 0.0f);
    e.colCdf.assign((size_t)e.H * (e.W + 1), 0.0f);
    for (int row = 0; row < e.H; row++) {
        float sinT = sinf(3.14159265358979323846f * (row + 0.5f) / e.H);
        float* cdf = &e.colCdf[(size_t)row * (e.W + 1)];
        cdf[0] = 0.f;
        for (int col = 0; col < e.W; col++) {
            const float* t = &e.rgba[((size_t)row * e.W + col) * 4];
            float lum = 0.2126f * t[0] + 0.7152f * t[1] + 0.0722f * t[2];
            cdf[col + 1] = cdf[col] + std::fmax(lum, 0.0f) * sinT;
        }
        e.rowCdf[row + 1] = e.rowCdf[row] + cdf[e.W];
    }
    e.total = e.rowCdf[e.H];
}

template <class T>
V<T> tex_bilinear(const Env& e, T u, T v) {
    T x = u * e.W - T(0.5), y = v * e.H - T(0.5);
    T fx = std::floor(x), fy = std::floor(y);
    T a = std::nearbyint((x - fx) * T(256)) / T(256), b = std::nearbyint((y - fy) * T(256)) / T(256);
    long long i0 = (long long)fx, j0 = (long long)fy;
    auto texel = [&](long long i, long long j) {
        i = ((i % e.W) + e.W) % e.W;
        j = std::min<long long>(std::max<long long>(j, 0), e.H - 1);
        const float* p = &e.rgba[((size_t)j * e.W + (size_t)i) * 4];
        return V<T>((T)p[0], (T)p[1], (T)p[2]);
    };
    return texel(i0, j0) * ((T(1) - a) * (T(1) - b)) + texel(i0 + 1, j0) * (a * (T(1) - b)) +
           texel(i0, j0 + 1) * ((T(1) - a) * b) + texel(i0 + 1, j0 + 1) * (a * b);
}

template <class T>
void env_uv(const Env& e, const V<T>& d, T& u, T& v) {
    const T PI = (T)kPiD;
    u = std::atan2(d.z, d.x) / (T(2) * PI) + T(0.5) + (T)e.rotation / (T(2) * PI);
    v = std::acos(std::fmin(std::fmax(d.y, T(-1)), T(1))) / PI;
    u = u - std::floor(u);
}

template <class T>
V<T> env_radiance(const Env& e, const V<T>& d, const V<T>& fallback) {
    if (!e.enabled) return fallback;
    T u, v;
    env_uv(e, d.norm(), u, v);
    return tex_bilinear(e, u, v) * (T)e.intensity;
}

template <class T>
T env_sel_prob(const Env& e, int lights) {
    if (!e.enabled || e.total <= 0.f) return T(0);
    return lights > 0 ? T(0.5) : T(1);
}

int find_cdf(const float* cdf, int count, float value) {
    int lo = 0, hi = count - 1;
    while (lo < hi) {
        int m = (lo + hi) >> 1;
        if (cdf[m + 1] <= value) lo = m + 1;
        else hi = m;
    }
    return lo;
}

template <class T>
T env_texel_pdf(const Env& e, int row, int col, T sinT) {
    if (sinT < T(1e-6f)) return T(0);
    const float* cdf = &e.colCdf[(size_t)row * (e.W + 1)];
    T w = (T)cdf[col + 1] - (T)cdf[col];
    const T PI = (T)kPiD;
    return w * e.W * e.H / ((T)e.total * T(2) * PI * PI * sinT);
}

template <class T>
T env_dir_pdf(const Env& e, const V<T>& d) {
    V<T> u = d.norm();
    T uu, vv;
    env_uv(e, u, uu, vv);
    int col = std::min((int)(uu * e.W), e.W - 1), row = std::min((int)(vv * e.H), e.H - 1);
    return env_texel_pdf<T>(e, row, col, std::sqrt(std::fmax(T(1) - u.y * u.y, T(0))));
}

template <class T>
V<T> env_sample(const Env& e, Rng& rng, T& pdf) {
    const T PI = (T)kPiD;
    int row = find_cdf(e.rowCdf.data(), e.H, rng.uniform() * e.total);
    const float* cdf = &e.colCdf[(size_t)row * (e.W + 1)];
    int col = find_cdf(cdf, e.W, rng.uniform() * cdf[e.W]);
    T u = ((T)col + (T)rng.uniform()) / e.W;
    T v = ((T)row + (T)rng.uniform()) / e.H;
    pdf = env_texel_pdf<T>(e, row, col, std::sin(v * PI));
    T phi = (u - T(0.5)) * T(2) * PI - (T)e.rotation, theta = v * PI, s = std::sin(theta);
    return V<T>(std::cos(phi) * s, std::cos(theta), std::sin(phi) * s);
}

// ---------------------------------------------------------------------------
// Integrator (PT:2874-3059 megakernel; the wavefront kernels PT:3342-3755
// evaluate the same estimator with the same draw order).
// ---------------------------------------------------------------------------
struct Scene {
    std::vector<mc_triangle> tris;
    std::vector<mc_triangle_hot> hot;
    std::vector<mc_sphere> sph;
    std::vector<mc_light> lights;
    Bvh bvh;
    Env env;
};

template <class T>
V<T> random_unit_vector(Rng& rng) {
    while (true) {
        T x = (T)(rng.uniform() * 2.f - 1.f), y = (T)(rng.uniform() * 2.f - 1.f), z = (T)(rng.uniform() * 2.f - 1.f);
        V<T> p(x, y, z);
        if (p.len2() < T(1)) return p.norm();
    }
}

template <class T>
V<T> refract(const V<T>& in, const V<T>& n, T eta) {  // PT:141-156
    V<T> d = in.norm();
    T c1 = std::fmin((-d).dot(n), T(1));
    T th1 = std::acos(c1);
    T s2 = std::sin(th1) * eta;
    if (s2 > T(1)) return d.reflect(n);
    T th2 = std::asin(s2);
    V<T> tang = d + n * c1;
    T tl = tang.len();
    if (tl > T(1e-8f)) tang = tang / tl;
    return tang * std::sin(th2) - n * std::cos(th2);
}

template <class T>
T hg_pdf(T c, T g) {  // PT:776-780
    T g2 = g * g, den = std::fmax(T(1) + g2 - T(2) * g * c, T(1e-6f));
    return (T(1) - g2) / (T(4) * (T)kPiD * den * std::sqrt(den));
}

template <class T>
T power_h(T a, T b) { return a * a / (a * a + b * b); }

struct MatInfo {
    int type;
    const mc_material* m;
};

template <class T>
void hit_geometry(const Scene& S, int type, int prim, const V<T>& o, const V<T>& d, T t, T time, V<T>& p, V<T>& normal,
                  bool& front, V<T>& albedo, const mc_material*& mat) {
    const T PI = (T)kPiD;
    T u = T(0), v = T(0);  // texture coordinates of the hit
    p = o + d * t;
    if (type == 0) {
        const mc_sphere& s = S.sph[prim];
        V<T> c = s.is_moving ? vin<T>(s.center) + (vin<T>(s.center1) - vin<T>(s.center)) * time : vin<T>(s.center);
        V<T> ow = (p - c).norm();
        front = d.dot(ow) < T(0);
        normal = front ? ow : -ow;
        mat = &s.mat;
        // PT:1505-1507 computeSphereUvFromOutwardNormal
        u = (std::atan2(-ow.z, ow.x) + PI) / (T(2) * PI);
        v = std::acos(std::fmin(T(1), std::fmax(T(-1), -ow.y))) / PI;
    } else {
        const mc_triangle& tr = S.tris[prim];
        V<T> v0 = vin<T>(tr.v0), v1 = vin<T>(tr.v1), v2 = vin<T>(tr.v2);
        V<T> fn = (v1 - v0).cross(v2 - v0).norm();
        front = d.dot(fn) < T(0);
        V<T> sn = fn;
        if (vin<T>(tr.n0).len2() != T(0)) {  // PT:697-713
            T a2 = (v1 - v0).cross(v2 - v0).len();
            T w0 = (v1 - p).cross(v2 - p).len() / a2, w1 = (v0 - p).cross(v2 - p).len() / a2, w2 = (v1 - p).cross(v0 - p).len() / a2;
            T ws = w0 + w1 + w2;
            if (ws > T(0) && ws <= T(1.01f)) {
                V<T> s = vin<T>(tr.n0) * w0 + vin<T>(tr.n1) * w1 + vin<T>(tr.n2) * w2;
                if (s.len2() >= T(1e-12f)) {
                    s = s.norm();
                    if (s.dot(fn) < T(0)) s = -s;
                    sn = s;
                }
            }
        }
        normal = front ? sn : -sn;
        mat = &tr.mat;
        // PT:687-695 computeTriangleUvFromHitPoint: area weights of the hit point
        const T a2 = (v1 - v0).cross(v2 - v0).len();
        const T w0 = (v1 - p).cross(v2 - p).len() / a2, w1 = (v0 - p).cross(v2 - p).len() / a2,
                w2 = (v1 - p).cross(v0 - p).len() / a2;
        u = (T)tr.uv0.x * w0 + (T)tr.uv1.x * w1 + (T)tr.uv2.x * w2;
        v = (T)tr.uv0.y * w0 + (T)tr.uv1.y * w1 + (T)tr.uv2.y * w2;
    }
    // PT:216-234 sampleTexture: solid, or a checker of (u, v) cells; image
    // textures are sampled by the GPU texture unit and are not restated here
    const mc_texture& tex = mat->albedo;
    albedo = vin<T>(tex.color_a);
    if (tex.type == MC_TEX_CHECKER) {
        const long long iu = (long long)std::floor(u * (T)tex.scale), iv = (long long)std::floor(v * (T)tex.scale);
        if (((iu + iv) & 1) != 0) albedo = vin<T>(tex.color_b);
    }
}

// mediumTransmittance (PT:2874-2898), homogeneous media only
template <class T>
T transmittance(const Scene& S, V<T> o, const V<T>& d, T time, T maxD) {
    T tr = T(1), travelled = T(0);
    for (int c = 0; c < 4; c++) {
        T rem = maxD - travelled;
        if (rem <= T(0)) break;
        T t;
        bool occ;
        int h = traverse<T>(S.bvh, S.hot.data(), S.sph.data(), o, d, time, rem, false, t, occ);
        if (h < 0) break;
        int type = h >> 30, prim = h & ((1 << 30) - 1);
        const mc_material& m = type == 0 ? S.sph[prim].mat : S.tris[prim].mat;
        if (m.type != MC_MAT_ISOTROPIC) return T(0);
        V<T> p, nn, alb;
        bool front;
        const mc_material* mm;
        hit_geometry<T>(S, type, prim, o, d, t, time, p, nn, front, alb, mm);
        if (!front) tr = tr * std::exp(-(T)m.density * t);
        travelled = travelled + t;
        o = p;
    }
    return tr;
}

template <class T>
void trace_path(const Scene& S, const mc_camera& cam, int px, int py, Rng& rng, int maxDepth, bool clamp, V<T>& out,
                double& ext, double& shd) {
    const T PI = (T)kPiD;
    // Camera::getRay (PT:1648-1658)
    V<T> pc = vin<T>(cam.pixel00) + vin<T>(cam.pixel_delta_u) * (T)px + vin<T>(cam.pixel_delta_v) * (T)py;
    V<T> lens;
    while (true) {
        T x = (T)(rng.uniform() * 2.f - 1.f), y = (T)(rng.uniform() * 2.f - 1.f);
        if (x * x + y * y < T(1)) { lens = V<T>(x, y, 0); break; }
    }
    lens = lens * (T)cam.lens_radius;
    V<T> o = vin<T>(cam.center) + vin<T>(cam.u) * lens.x + vin<T>(cam.v) * lens.y;
    T time = (T)rng.uniform();
    V<T> d = (pc - o).norm();
    V<T> att(1, 1, 1), col(0, 0, 0);
    bool prevSpec = true;
    T prevPdf = T(1);
    const int L = (int)S.lights.size();
    const T envP = env_sel_prob<T>(S.env, L);
    for (int depth = 0; depth < maxDepth; depth++) {
        ext += 1;
        T t;
        bool occ;
        int h = traverse<T>(S.bvh, S.hot.data(), S.sph.data(), o, d, time, T(1e30f), false, t, occ);
        if (h < 0) {
            T w = T(1);
            if (!(depth == 0 || prevSpec) && envP > T(0)) w = power_h<T>(prevPdf, envP * env_dir_pdf<T>(S.env, d));
            col = col + att * env_radiance<T>(S.env, d, vin<T>(cam.background)) * w;
            break;
        }
        int type = h >> 30, prim = h & ((1 << 30) - 1);
        V<T> p, n, alb;
        bool front;
        const mc_material* m;
        hit_geometry<T>(S, type, prim, o, d, t, time, p, n, front, alb, m);
        if (m->type == MC_MAT_EMISSIVE) {
            T w = T(1);
            if (!(depth == 0 || prevSpec) && type == 1) {
                T cosL = std::fmax(std::fabs(d.dot(n)), T(1e-4f));
                const mc_triangle& tr = S.tris[prim];
                T area = T(0.5) * (vin<T>(tr.v1) - vin<T>(tr.v0)).cross(vin<T>(tr.v2) - vin<T>(tr.v0)).len();
                T lp = ((T(1) - envP) / (T)L) * (t * t) / (cosL * area);
                w = power_h<T>(prevPdf, lp);
            }
            col = col + att * vin<T>(m->emitted) * w;
            break;
        }
        V<T> so = p;
        if (m->type == MC_MAT_ISOTROPIC) {
            T sd = front ? t : -std::log(T(1) - (T)rng.uniform()) / (T)m->density;
            if (sd >= t) {
                o = p;
                continue;
            }
            so = o + d * sd;
        }
        att = att * alb;
        if ((m->type == MC_MAT_LAMBERTIAN || m->type == MC_MAT_ISOTROPIC) && (L > 0 || envP > T(0))) {
            V<T> tl, lc;
            T dist, sp;
            if (envP > T(0) && (L == 0 || (T)rng.uniform() < envP)) {
                T dp;
                tl = env_sample<T>(S.env, rng, dp);
                lc = env_radiance<T>(S.env, tl, V<T>(0, 0, 0));
                dist = T(1e30f);
                sp = envP * dp;
            } else {
                int li = std::min((int)(rng.uniform() * L), L - 1);
                const mc_light& lt = S.lights[li];
                T sel = (T(1) - envP) / (T)L;
                T r1 = (T)rng.uniform(), r2 = (T)rng.uniform(), s1 = std::sqrt(r1);
                T w0 = T(1) - s1, w1 = r2 * s1, w2 = T(1) - w0 - w1;
                V<T> pt = vin<T>(lt.tri.v0) * w0 + vin<T>(lt.tri.v1) * w1 + vin<T>(lt.tri.v2) * w2;
                V<T> vec = pt - so;
                dist = vec.len();
                tl = vec / dist;
                lc = vin<T>(lt.emitted);
                T cl = std::fabs(vin<T>(lt.normal).dot(tl));
                sp = cl > T(1e-4f) ? sel * (dist * dist) / (cl * (T)lt.area) : T(0);
            }
            bool iso = m->type == MC_MAT_ISOTROPIC;
            T cs = iso ? T(1) : n.dot(tl);
            if (cs > T(0) && sp > T(0)) {
                shd += 1;
                T tr = transmittance<T>(S, so, tl, time, dist * T(0.999f));
                if (tr > T(0)) {
                    T ph = hg_pdf<T>(d.dot(tl), (T)m->phase_g);
                    T spdf = iso ? ph : cs / PI;
                    T sval = iso ? ph : cs / PI;
                    T w = power_h<T>(sp, spdf);
                    col = col + att * lc * (sval / sp) * w * tr;
                }
            }
        }
        if (depth > 3) {
            T mx = std::fmax(att.x, std::fmax(att.y, att.z));
            T cont = std::fmin(mx, (T)cam.rr_cap);
            if ((T)rng.uniform() > cont) break;
            att = att / cont;
        }
        V<T> nd;
        switch (m->type) {
            case MC_MAT_CONDUCTOR: nd = (d.norm().reflect(n) + random_unit_vector<T>(rng) * (T)m->fuzz).norm(); break;
            case MC_MAT_DIELECTRIC: {
                T eta = front ? T(1) / (T)m->refraction_index : (T)m->refraction_index;
                V<T> u = d.norm();
                T c = std::fmin((-u).dot(n), T(1)), s = std::sqrt(T(1) - c * c);
                T r0 = (T(1) - eta) / (T(1) + eta);
                r0 = r0 * r0;
                T rp = (eta * s > T(1)) ? T(1) : r0 + (T(1) - r0) * std::pow(T(1) - c, T(5));
                nd = ((T)rng.uniform() < rp) ? u.reflect(n) : refract<T>(u, n, eta);
                break;
            }
            case MC_MAT_ISOTROPIC: {
                T g = (T)m->phase_g;
                if (std::fabs(g) < T(1e-3f)) {
                    T u1 = (T)rng.uniform(), u2 = (T)rng.uniform();
                    T z = T(1) - T(2) * u1, r = std::sqrt(std::fmax(T(0), T(1) - z * z)), ph = T(2) * PI * u2;
                    nd = V<T>(r * std::cos(ph), r * std::sin(ph), z);
                } else {
                    T u1 = (T)rng.uniform(), u2 = (T)rng.uniform();
                    T sq = (T(1) - g * g) / (T(1) + g - T(2) * g * u1);
                    T ct = std::fmin(std::fmax((T(1) + g * g - sq * sq) / (T(2) * g), T(-1)), T(1));
                    T st = std::sqrt(std::fmax(T(0), T(1) - ct * ct)), ph = T(2) * PI * u2;
                    V<T> f = d.norm();
                    V<T> hlp = std::fabs(f.x) > T(0.9f) ? V<T>(0, 1, 0) : V<T>(1, 0, 0);
                    V<T> ta = hlp.cross(f).norm(), bt = f.cross(ta);
                    nd = ta * (st * std::cos(ph)) + bt * (st * std::sin(ph)) + f * ct;
                }
                break;
            }
            default: {
                V<T> r = n + random_unit_vector<T>(rng);
                nd = r.len2() < T(1e-8f) ? n : r.norm();
            }
        }
        prevSpec = m->type != MC_MAT_LAMBERTIAN && m->type != MC_MAT_ISOTROPIC;
        prevPdf = m->type == MC_MAT_ISOTROPIC ? hg_pdf<T>(d.dot(nd), (T)m->phase_g) : std::fmax(nd.dot(n), T(0)) / PI;
        o = so;
        d = nd;
    }
    if (clamp) {
        T b = std::fmax(col.x, std::fmax(col.y, col.z));
        if (b > T(10)) col = col * (T(10) / b);
    }
    out = col;
}

}  // namespace

extern "C" {

void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c[4] = {ctr[0], ctr[1], ctr[2], ctr[3]};
    philox(c, key[0], key[1]);
    for (int i = 0; i < 4; i++) out[i] = c[i];
}

int orc_finalize_sort(const mc_triangle* tris, int nt, const mc_sphere* sph, int ns, uint32_t* codes_ref_order,
                      uint32_t* sorted_codes, int32_t* perm, mc_aabb* bounds_ref_order, mc_aabb* scene_bounds) {
    int n = nt + ns;
    if (n <= 0) return 1;
    std::vector<Box> boxes(n);
    std::vector<float> cent((size_t)n * 3);
    for (int i = 0; i < n; i++) prim_box(tris, sph, ns, i, boxes[i], &cent[(size_t)i * 3]);
    Box sb = boxes[0];
    for (int i = 1; i < n; i++) sb = merge(sb, boxes[i]);  // PT:1937-1946, spheres then triangles
    struct Ref {
        uint32_t code;
        int32_t idx;
    };
    std::vector<Ref> refs(n);
    for (int i = 0; i < n; i++) {
        uint32_t x = expand_bits(quantize(cent[i * 3 + 0], sb.lx, sb.hx));
        uint32_t y = expand_bits(quantize(cent[i * 3 + 1], sb.ly, sb.hy));
        uint32_t z = expand_bits(quantize(cent[i * 3 + 2], sb.lz, sb.hz));
        refs[i] = Ref{x | y << 1 | z << 2, i};
        if (codes_ref_order) codes_ref_order[i] = refs[i].code;
        if (bounds_ref_order) bounds_ref_order[i] = to_aabb(boxes[i]);
    }
    // the reference sorts with std::sort and a strict less-than on the code (PT:4224-4226)
    std::sort(refs.begin(), refs.end(), [](const Ref& a, const Ref& b) { return a.code < b.code; });
    for (int k = 0; k < n; k++) {
        if (sorted_codes) sorted_codes[k] = refs[k].code;
        if (perm) perm[k] = refs[k].idx;
    }
    if (scene_bounds) *scene_bounds = to_aabb(sb);
    return 0;
}

int orc_build(const uint32_t* codes, const int32_t* perm, const mc_aabb* boxes, int n, int ns, mc_bvh_node* internal,
              mc_bvh_node* leaves) {
    if (n <= 0) return 1;
    for (int k = 0; k < n; k++) {
        mc_bvh_node& l = leaves[k];
        std::memset(&l, 0, sizeof(l));
        l.bounds = boxes[perm[k]];
        l.prim = perm[k] < ns ? perm[k] : perm[k] - ns;
        l.is_leaf = 1;
        l.left = l.right = -1;
        l.parent = -1;
    }
    if (n == 1) return 0;
    for (int i = 0; i < n - 1; i++) std::memset(&internal[i], 0, sizeof(mc_bvh_node));
    for (int i = 0; i < n - 1; i++) {
        int lft, rgt;
        bool ll, rl;
        karras(codes, n, i, lft, rgt, ll, rl);
        mc_bvh_node& nd = internal[i];
        nd.left = lft;
        nd.right = rgt;
        nd.left_is_leaf = ll;
        nd.right_is_leaf = rl;
        nd.prim = -1;
        (ll ? leaves[lft] : internal[lft]).parent = i;
        (rl ? leaves[rgt] : internal[rgt]).parent = i;
    }
    internal[0].parent = -1;
    // refit: post-order over the hierarchy (PT:1398-1415 computes the same merges bottom-up)
    std::vector<int> stack;
    std::vector<char> state(n - 1, 0);
    stack.push_back(0);
    while (!stack.empty()) {
        int i = stack.back();
        mc_bvh_node& nd = internal[i];
        if (state[i] == 0) {
            state[i] = 1;
            if (!nd.right_is_leaf) stack.push_back(nd.right);
            if (!nd.left_is_leaf) stack.push_back(nd.left);
            continue;
        }
        stack.pop_back();
        const mc_aabb& a = nd.left_is_leaf ? leaves[nd.left].bounds : internal[nd.left].bounds;
        const mc_aabb& b = nd.right_is_leaf ? leaves[nd.right].bounds : internal[nd.right].bounds;
        nd.bounds = to_aabb(merge(from_aabb(a), from_aabb(b)));
    }
    return 0;
}

int orc_depth(const mc_bvh_node* internal, const mc_bvh_node* leaves, int n) {
    int best = 0;
    for (int k = 0; k < n; k++) {
        int d = 0, p = leaves[k].parent;
        while (p >= 0 && d <= n) {
            d++;
            p = internal[p].parent;
        }
        best = std::max(best, d);
    }
    return best;
}

int orc_trace(const mc_bvh_node* internal, const mc_bvh_node* leaves, const int32_t* leaf_types, int n,
              const mc_triangle_hot* hot, const mc_sphere* sph, const float* rays, int nr, int mode, const float* tmax,
              mc_packed_hit* hits, int32_t* occluded, int threads) {
    Bvh b;
    b.n = n;
    b.internal.assign(internal, internal + std::max(0, n - 1));
    if (n == 1) b.internal.resize(1);
    b.leaves.assign(leaves, leaves + n);
    b.types.assign(leaf_types, leaf_types + n);
    threads = std::max(1, threads);
    std::atomic<int> next(0);
    auto work = [&]() {
        const int chunk = 1024;
        for (int s = next.fetch_add(chunk); s < nr; s = next.fetch_add(chunk)) {
            for (int i = s; i < std::min(nr, s + chunk); i++) {
                V<float> o(rays[i], rays[nr + i], rays[2 * (size_t)nr + i]);
                V<float> d(rays[3 * (size_t)nr + i], rays[4 * (size_t)nr + i], rays[5 * (size_t)nr + i]);
                float time = rays[6 * (size_t)nr + i];
                float t;
                bool occ;
                if (mode == 0) {
                    int h = traverse<float>(b, hot, sph, o, d, time, 1e30f, false, t, occ);
                    hits[i].t = t;
                    hits[i].type = h < 0 ? -1 : (h >> 30);
                    hits[i].index = h < 0 ? -1 : (h & ((1 << 30) - 1));
                    hits[i].did_hit = h < 0 ? 0 : 1;
                } else {
                    traverse<float>(b, hot, sph, o, d, time, tmax[i], true, t, occ);
                    occluded[i] = occ ? 1 : 0;
                }
            }
        }
    };
    std::vector<std::thread> pool;
    for (int i = 1; i < threads; i++) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
    return 0;
}

void* orc_scene_create(const mc_triangle* tris, int nt, const mc_sphere* sph, int ns, const float* env_rgba, int env_w,
                       int env_h, float env_intensity, float env_rotation) {
    if (nt + ns <= 0) return nullptr;
    Scene* S = new Scene();
    S->tris.assign(tris, tris + nt);
    S->sph.assign(sph, sph + ns);
    S->hot.resize(nt);
    for (int i = 0; i < nt; i++) {
        const mc_triangle& t = tris[i];
        S->hot[i].v0 = t.v0; S->hot[i].v1 = t.v1; S->hot[i].v2 = t.v2;
        if (t.mat.type == MC_MAT_EMISSIVE) {  // PT:1972-1985
            V<float> v0 = vin<float>(t.v0), v1 = vin<float>(t.v1), v2 = vin<float>(t.v2);
            V<float> a = (v1 - v0).cross(v2 - v0);
            mc_light L;
            L.tri = S->hot[i];
            L.emitted = t.mat.emitted;
            L.area = 0.5f * a.len();
            V<float> nn = a.norm();
            L.normal = mc_vec3{nn.x, nn.y, nn.z};
            S->lights.push_back(L);
        }
    }
    build_bvh(tris, nt, sph, ns, S->bvh);
    if (env_rgba && env_w > 0 && env_h > 0) {
        S->env.enabled = true;
        S->env.W = env_w;
        S->env.H = env_h;
        S->env.rgba.assign(env_rgba, env_rgba + (size_t)env_w * env_h * 4);
        env_tables(S->env);
    }
    S->env.intensity = env_intensity;
    S->env.rotation = env_rotation;
    return S;
}

void orc_scene_destroy(void* s) { delete (Scene*)s; }

int orc_render(void* scene, const mc_camera* cam, int W, int H, int spp, int first_sample, int max_depth, uint64_t seed,
               int use_double, int disable_clamp, int x0, int y0, int x1, int y1, int threads, double* accum,
               double* stats) {
    if (!scene || !cam || !accum || W <= 0 || H <= 0) return 1;
    const Scene& S = *(const Scene*)scene;
    x0 = std::max(0, x0); y0 = std::max(0, y0); x1 = std::min(W, x1); y1 = std::min(H, y1);
    threads = std::max(1, threads);
    std::atomic<int> nextRow(y0);
    std::vector<double> ext(threads, 0.0), shd(threads, 0.0);
    auto work = [&](int tid) {
        for (int y = nextRow++; y < y1; y = nextRow++) {
            for (int x = x0; x < x1; x++) {
                int pixel = y * W + x;
                for (int s = 0; s < spp; s++) {
                    Rng rng{(uint32_t)seed, (uint32_t)(seed >> 32), (uint32_t)(first_sample + s), (uint32_t)pixel, 0u};
                    double r, g, b;
                    if (use_double) {
                        V<double> c;
                        trace_path<double>(S, *cam, x, y, rng, max_depth, !disable_clamp, c, ext[tid], shd[tid]);
                        r = c.x; g = c.y; b = c.z;
                    } else {
                        V<float> c;
                        trace_path<float>(S, *cam, x, y, rng, max_depth, !disable_clamp, c, ext[tid], shd[tid]);
                        r = c.x; g = c.y; b = c.z;
                    }
                    accum[(size_t)pixel * 3 + 0] += r;
                    accum[(size_t)pixel * 3 + 1] += g;
                    accum[(size_t)pixel * 3 + 2] += b;
                }
            }
        }
    };
    std::vector<std::thread> pool;
    for (int i = 1; i < threads; i++) pool.emplace_back(work, i);
    work(0);
    for (auto& t : pool) t.join();
    if (stats) {
        stats[0] = stats[1] = 0;
        for (int i = 0; i < threads; i++) { stats[0] += ext[i]; stats[1] += shd[i]; }
    }
    return 0;
}

}  // extern "C"
