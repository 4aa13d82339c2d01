// mc_scene_gen.cpp - the seeded synthetic scenes the benchmarks and tests
// render, and the host scene helpers they are built from (quads, boxes,
// spheres, the camera set-up, triangle bounds and the light list).
//
// Host-only code with no dependency on the rest of the library (mc_abi.h
// types and mc_host_scene.h only), so that any program that must render the
// same scenes can compile this one file and obtain byte-identical triangles.
// Compiled by the host compiler with -O2 -ffp-contract=off -fno-fast-math: the
// reference runs the camera set-up and finalizeScene on the host (PT:1610-1631,
// 1930-1987), so the float results are bit-identical when the operations are
// written in the same order.
#include "mc_scene_gen.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

namespace mc_gen {

using namespace mc_host;

// PT:1610-1631 Camera::initialize, in the same operation order on the host.
void camera_initialize(mc_camera& c) {
    mc_camera* cam = &c;
    HV look_from(cam->look_from), look_at(cam->look_at), up(cam->up);
    HV w = (look_from - look_at).normalize();
    HV u = up.cross(w).normalize();
    HV v = w.cross(u);
    cam->lens_radius = cam->aperture / 2.;
    cam->image_height = int(cam->image_width / cam->aspect_ratio);
    HV center = look_from;
    float theta = cam->vfov * (3.14159265358979323846f / 180.0f);
    float h = tanf(theta / 2.0f);
    float viewport_height = 2.0f * h * cam->focus_distance;
    float viewport_width = viewport_height * (float(cam->image_width) / cam->image_height);
    HV viewport_u = u * viewport_width;
    HV viewport_v = v * -viewport_height;
    HV pdu = viewport_u / float(cam->image_width);
    HV pdv = viewport_v / float(cam->image_height);
    HV upper_left = center - (w * cam->focus_distance) - viewport_u / 2.0f - viewport_v / 2.0f;
    HV p00 = upper_left + (pdu + pdv) * 0.5f;
    cam->w = w; cam->u = u; cam->v = v;
    cam->center = center;
    cam->pixel_delta_u = pdu;
    cam->pixel_delta_v = pdv;
    cam->pixel00 = p00;
}

// PT:651-655 calculate_bounding_box for each triangle and PT:1972-1985 light list.
void finalize(mc_triangle* tris, int32_t n, mc_light* lights, int32_t* light_count) {
    const float eps = 1e-3f;
    int32_t nl = 0;
    for (int32_t i = 0; i < n; i++) {
        mc_triangle& t = tris[i];
        t.aabb.lo = mc_vec3{fminf(t.v0.x, fminf(t.v1.x, t.v2.x)) - eps, fminf(t.v0.y, fminf(t.v1.y, t.v2.y)) - eps,
                            fminf(t.v0.z, fminf(t.v1.z, t.v2.z)) - eps};
        t.aabb.hi = mc_vec3{fmaxf(t.v0.x, fmaxf(t.v1.x, t.v2.x)) + eps, fmaxf(t.v0.y, fmaxf(t.v1.y, t.v2.y)) + eps,
                            fmaxf(t.v0.z, fmaxf(t.v1.z, t.v2.z)) + eps};
        t.aabb.pad0 = 0.f;
        t.aabb.pad1 = 0.f;
        if (t.mat.type == MC_MAT_EMISSIVE) {
            HV v0(t.v0), v1(t.v1), v2(t.v2);
            HV area = (v1 - v0).cross(v2 - v0);
            if (lights) {
                mc_light& L = lights[nl];
                L.tri.v0 = t.v0; L.tri.v1 = t.v1; L.tri.v2 = t.v2;
                L.emitted = t.mat.emitted;
                L.area = 0.5f * area.length();
                L.normal = area.normalize();
            }
            nl++;
        }
    }
    if (light_count) *light_count = nl;
}


// PT:1677-1691 add_quad
void add_quad(std::vector<mc_triangle>& tris, HV a, HV b, HV c, HV d, const mc_material& m) {
    mc_triangle t0 = make_triangle(a, b, c, m);
    mc_triangle t1 = make_triangle(a, c, d, m);
    t0.uv0 = mc_vec2{0.f, 0.f}; t0.uv1 = mc_vec2{1.f, 0.f}; t0.uv2 = mc_vec2{1.f, 1.f};
    t1.uv0 = mc_vec2{0.f, 0.f}; t1.uv1 = mc_vec2{1.f, 1.f}; t1.uv2 = mc_vec2{0.f, 1.f};
    tris.push_back(t0);
    tris.push_back(t1);
}

// PT:1693-1708 add_box
void add_box(std::vector<mc_triangle>& tris, HV center, HV half, float rotY, const mc_material& m) {
    float cs = cosf(rotY), sn = sinf(rotY);
    HV p[8];
    for (int i = 0; i < 8; i++) {
        float x = (i & 1) ? half.x : -half.x;
        float y = (i & 2) ? half.y : -half.y;
        float z = (i & 4) ? half.z : -half.z;
        p[i] = center + HV(x * cs + z * sn, y, -x * sn + z * cs);
    }
    add_quad(tris, p[0], p[1], p[3], p[2], m);
    add_quad(tris, p[4], p[5], p[7], p[6], m);
    add_quad(tris, p[0], p[2], p[6], p[4], m);
    add_quad(tris, p[1], p[3], p[7], p[5], m);
    add_quad(tris, p[0], p[1], p[5], p[4], m);
    add_quad(tris, p[2], p[3], p[7], p[6], m);
}

// ---------------------------------------------------------------------------
// Seeded generators. SplitMix64 for all draws (Steele, Lea, Flood 2014).
// ---------------------------------------------------------------------------
struct SplitMix {
    uint64_t s;
    explicit SplitMix(uint64_t seed) : s(seed) {}
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
    double normal() {
        double u1 = uniform(), u2 = uniform();
        if (u1 < 1e-300) u1 = 1e-300;
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * M_PI * u2);
    }
};

uint32_t hash3(int x, int y, int z, uint32_t seed) {
    uint32_t h = seed * 0x9E3779B1u;
    h ^= (uint32_t)x * 0x85EBCA77u;
    h = (h << 13) | (h >> 19);
    h ^= (uint32_t)y * 0xC2B2AE3Du;
    h = (h << 17) | (h >> 15);
    h ^= (uint32_t)z * 0x27D4EB2Fu;
    h ^= h >> 15;
    h *= 0x2C1B3C6Du;
    h ^= h >> 12;
    h *= 0x297A2D39u;
    h ^= h >> 15;
    return h;
}

// Value noise on the integer lattice, smoothstep-weighted trilinear blend, in [-1, 1].
double value_noise(double x, double y, double z, uint32_t seed) {
    double fx = std::floor(x), fy = std::floor(y), fz = std::floor(z);
    int ix = (int)fx, iy = (int)fy, iz = (int)fz;
    double tx = x - fx, ty = y - fy, tz = z - fz;
    tx = tx * tx * (3 - 2 * tx);
    ty = ty * ty * (3 - 2 * ty);
    tz = tz * tz * (3 - 2 * tz);
    double c[8];
    for (int i = 0; i < 8; i++) {
        uint32_t h = hash3(ix + (i & 1), iy + ((i >> 1) & 1), iz + ((i >> 2) & 1), seed);
        c[i] = (double)h * (2.0 / 4294967295.0) - 1.0;
    }
    double x00 = c[0] + (c[1] - c[0]) * tx, x10 = c[2] + (c[3] - c[2]) * tx;
    double x01 = c[4] + (c[5] - c[4]) * tx, x11 = c[6] + (c[7] - c[6]) * tx;
    double y0 = x00 + (x10 - x00) * ty, y1 = x01 + (x11 - x01) * ty;
    return y0 + (y1 - y0) * tz;
}

// 4-octave fractional Brownian motion of value noise, normalized to [-1, 1].
double fbm4(double x, double y, double z, uint32_t seed) {
    double sum = 0, amp = 1, norm = 0, f = 1;
    for (int o = 0; o < 4; o++) {
        sum += amp * value_noise(x * f, y * f, z * f, seed + 101u * (uint32_t)o);
        norm += amp;
        amp *= 0.5;
        f *= 2.0;
    }
    return sum / norm;
}

struct DV { double x, y, z; };
DV dnorm(DV a) {
    double l = std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z);
    return DV{a.x / l, a.y / l, a.z / l};
}
DV dmid(DV a, DV b) { return dnorm(DV{a.x + b.x, a.y + b.y, a.z + b.z}); }

struct Xform {
    double r[3][3];
    DV t;
    double scale;
    DV apply(DV p) const {
        return DV{(r[0][0] * p.x + r[0][1] * p.y + r[0][2] * p.z) * scale + t.x,
                  (r[1][0] * p.x + r[1][1] * p.y + r[1][2] * p.z) * scale + t.y,
                  (r[2][0] * p.x + r[2][1] * p.y + r[2][2] * p.z) * scale + t.z};
    }
};

// Uniform random rotation from a random unit quaternion (Shoemake 1992).
Xform random_rotation(SplitMix& rng) {
    double u1 = rng.uniform(), u2 = rng.uniform(), u3 = rng.uniform();
    double a = std::sqrt(1 - u1), b = std::sqrt(u1);
    double qx = a * std::sin(2 * M_PI * u2), qy = a * std::cos(2 * M_PI * u2);
    double qz = b * std::sin(2 * M_PI * u3), qw = b * std::cos(2 * M_PI * u3);
    Xform x;
    x.r[0][0] = 1 - 2 * (qy * qy + qz * qz); x.r[0][1] = 2 * (qx * qy - qz * qw); x.r[0][2] = 2 * (qx * qz + qy * qw);
    x.r[1][0] = 2 * (qx * qy + qz * qw); x.r[1][1] = 1 - 2 * (qx * qx + qz * qz); x.r[1][2] = 2 * (qy * qz - qx * qw);
    x.r[2][0] = 2 * (qx * qz - qy * qw); x.r[2][1] = 2 * (qy * qz + qx * qw); x.r[2][2] = 1 - 2 * (qx * qx + qy * qy);
    x.t = DV{0, 0, 0};
    x.scale = 1;
    return x;
}

const double kPhi = 1.6180339887498948482;
const DV kIcoVerts[12] = {{-1, kPhi, 0}, {1, kPhi, 0}, {-1, -kPhi, 0}, {1, -kPhi, 0},
                          {0, -1, kPhi}, {0, 1, kPhi}, {0, -1, -kPhi}, {0, 1, -kPhi},
                          {kPhi, 0, -1}, {kPhi, 0, 1}, {-kPhi, 0, -1}, {-kPhi, 0, 1}};
const int kIcoFaces[20][3] = {{0, 11, 5}, {0, 5, 1}, {0, 1, 7}, {0, 7, 10}, {0, 10, 11},
                              {1, 5, 9}, {5, 11, 4}, {11, 10, 2}, {10, 7, 6}, {7, 1, 8},
                              {3, 9, 4}, {3, 4, 2}, {3, 2, 6}, {3, 6, 8}, {3, 8, 9},
                              {4, 9, 5}, {2, 4, 11}, {6, 2, 10}, {8, 6, 7}, {9, 8, 1}};

struct Displace {
    double amplitude;
    double frequency;
    uint32_t seed;
    DV apply(DV u) const {
        double r = 1.0 + amplitude * fbm4(u.x * frequency, u.y * frequency, u.z * frequency, seed);
        return DV{u.x * r, u.y * r, u.z * r};
    }
};

void subdivide(DV a, DV b, DV c, int level, const Displace& disp, const Xform& xf, const mc_material& m,
               mc_triangle* out, size_t& k) {
    if (level == 0) {
        DV pa = xf.apply(disp.apply(a)), pb = xf.apply(disp.apply(b)), pc = xf.apply(disp.apply(c));
        out[k++] = make_triangle(HV((float)pa.x, (float)pa.y, (float)pa.z), HV((float)pb.x, (float)pb.y, (float)pb.z),
                                 HV((float)pc.x, (float)pc.y, (float)pc.z), m);
        return;
    }
    DV ab = dmid(a, b), bc = dmid(b, c), ca = dmid(c, a);
    subdivide(a, ab, ca, level - 1, disp, xf, m, out, k);
    subdivide(b, bc, ab, level - 1, disp, xf, m, out, k);
    subdivide(c, ca, bc, level - 1, disp, xf, m, out, k);
    subdivide(ab, bc, ca, level - 1, disp, xf, m, out, k);
}

// Appends a displaced icosphere of 20*4^level triangles (threads over the 20 base faces).
void add_icosphere(std::vector<mc_triangle>& tris, int level, const Displace& disp, const Xform& xf, const mc_material& m) {
    size_t perFace = (size_t)1 << (2 * level);
    size_t base = tris.size();
    tris.resize(base + 20 * perFace);
    mc_triangle* out = tris.data() + base;
    unsigned hw = std::max(1u, std::min(20u, std::thread::hardware_concurrency()));
    std::atomic<int> next(0);
    auto work = [&]() {
        for (int f = next++; f < 20; f = next++) {
            DV a = dnorm(kIcoVerts[kIcoFaces[f][0]]), b = dnorm(kIcoVerts[kIcoFaces[f][1]]), c = dnorm(kIcoVerts[kIcoFaces[f][2]]);
            size_t k = (size_t)f * perFace;
            subdivide(a, b, c, level, disp, xf, m, out, k);
        }
    };
    std::vector<std::thread> pool;
    for (unsigned i = 1; i < hw; i++) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
}

// The procedural sky of the reference's scripts/make_sky.py (gradient, ground
// colour below the horizon, a 2-degree sun at 50 degrees elevation and a soft
// glow), evaluated for any W x H, RGBA, top row first (the renderer's layout).
void make_sky(int W, int H, std::vector<float>& rgba) {
    rgba.assign((size_t)W * H * 4, 0.f);
    const double elev = 50.0 * M_PI / 180.0, azim = 30.0 * M_PI / 180.0;
    const double sun[3] = {std::cos(elev) * std::cos(azim), std::sin(elev), std::cos(elev) * std::sin(azim)};
    const double zen[3] = {0.20, 0.45, 1.00}, hor[3] = {0.90, 0.95, 1.00}, gnd[3] = {0.25, 0.22, 0.18};
    const double sunRad[3] = {600.0, 560.0, 480.0}, glow[3] = {1.2, 1.0, 0.7};
    for (int row = 0; row < H; row++) {
        double v = (row + 0.5) / H, theta = v * M_PI;
        double sinT = std::sin(theta), dy = std::cos(theta);
        for (int col = 0; col < W; col++) {
            double u = (col + 0.5) / W, phi = (u - 0.5) * 2 * M_PI;
            double dx = std::cos(phi) * sinT, dz = std::sin(phi) * sinT;
            double up = std::min(1.0, std::max(-1.0, dy));
            double t = std::sqrt(std::min(1.0, std::max(0.0, up)));
            double c[3];
            for (int k = 0; k < 3; k++) {
                double sky = hor[k] * (1 - t) + zen[k] * t;
                c[k] = (up >= 0 ? sky : gnd[k]) * 0.8;
            }
            double cosang = std::min(1.0, std::max(-1.0, dx * sun[0] + dy * sun[1] + dz * sun[2]));
            double ang = std::acos(cosang);
            double g = std::exp(-(ang / (12.0 * M_PI / 180.0)) * (ang / (12.0 * M_PI / 180.0)));
            for (int k = 0; k < 3; k++) c[k] += (ang < 2.0 * M_PI / 180.0 ? sunRad[k] : 0.0) + g * glow[k];
            float* px = &rgba[((size_t)row * W + col) * 4];
            px[0] = (float)c[0];
            px[1] = (float)c[1];
            px[2] = (float)c[2];
            px[3] = 1.0f;
        }
    }
}

void set_camera(mc_camera& cam, int W, int H, HV from, HV at, float vfov, float focus, int depth, int spp) {
    std::memset(&cam, 0, sizeof(cam));
    cam.aspect_ratio = W / float(H);
    cam.image_width = W;
    cam.samples_per_pixel = spp;
    cam.max_depth = depth;
    cam.vfov = vfov;
    cam.look_from = from;
    cam.look_at = at;
    cam.up = mc_vec3{0, 1, 0};
    cam.aperture = 0.f;
    cam.focus_distance = focus;
    cam.rr_cap = 0.95f;
    cam.background = mc_vec3{0, 0, 0};
    camera_initialize(cam);
}

// Config: "cornell_boxes" - buildCornellRoom (PT:1747-1763) with a white 0.73
// floor, the reference's tall box (PT:1772-1773) and a short box (centre
// (0.7, 0.6, -1.8), half 0.6, rotY -0.3). Camera as main() (PT:4114-4124).
void gen_cornell_boxes(mc_scene_host& s, std::vector<mc_triangle>& tris) {
    mc_material white = make_lambertian(HV(0.73f, 0.73f, 0.73f));
    mc_material red = make_lambertian(HV(0.65f, 0.05f, 0.05f));
    mc_material green = make_lambertian(HV(0.12f, 0.45f, 0.15f));
    mc_material light = make_emissive(HV(15.0f, 15.0f, 15.0f));
    const float L = -2.f, R = 2.f, B = 0.f, T = 4.f, F = -4.f, N = 0.f;
    add_quad(tris, HV(L, B, N), HV(R, B, N), HV(R, B, F), HV(L, B, F), white);
    add_quad(tris, HV(L, T, N), HV(R, T, N), HV(R, T, F), HV(L, T, F), white);
    add_quad(tris, HV(L, B, F), HV(R, B, F), HV(R, T, F), HV(L, T, F), white);
    add_quad(tris, HV(L, B, N), HV(L, B, F), HV(L, T, F), HV(L, T, N), red);
    add_quad(tris, HV(R, B, N), HV(R, B, F), HV(R, T, F), HV(R, T, N), green);
    add_quad(tris, HV(-1.f, T - 0.01f, -2.6f), HV(1.f, T - 0.01f, -2.6f), HV(1.f, T - 0.01f, -1.4f),
             HV(-1.f, T - 0.01f, -1.4f), light);
    add_box(tris, HV(-0.8f, 1.1f, -2.8f), HV(0.55f, 1.1f, 0.55f), 0.3f, white);
    add_box(tris, HV(0.7f, 0.6f, -1.8f), HV(0.6f, 0.6f, 0.6f), -0.3f, white);
    s.width = 512; s.height = 512; s.spp = 64; s.max_depth = 8;
    set_camera(s.camera, 512, 512, HV(0, 2, 5.5f), HV(0, 2, -2), 40.0f, 7.5f, 8, 64);
}

mc_sphere make_sphere(HV c0, HV c1, bool moving, float r, const mc_material& m) {
    mc_sphere s;
    std::memset(&s, 0, sizeof(s));
    s.center = c0;
    s.center1 = c1;
    s.is_moving = moving ? 1 : 0;
    s.radius = r;
    s.mat = m;
    HV rv(r, r, r);  // PT:850-859 calculate_bounding_box
    HV lo = c0 - rv, hi = c0 + rv;
    if (moving) {
        HV lo1 = c1 - rv, hi1 = c1 + rv;
        lo = HV(fminf(lo.x, lo1.x), fminf(lo.y, lo1.y), fminf(lo.z, lo1.z));
        hi = HV(fmaxf(hi.x, hi1.x), fmaxf(hi.y, hi1.y), fmaxf(hi.z, hi1.z));
    }
    s.aabb.lo = lo;
    s.aabb.hi = hi;
    return s;
}

// Scene "cornell_spheres": the reference's buildCornellScene (PT:1765-1822) —
// checker floor, tall box, mirror sphere, smoke sphere (homogeneous isotropic
// medium) and a 13x13 grid of small spheres (80% diffuse and moving, 15%
// conductor, 5% dielectric) — with a seeded generator in place of rand() and
// without the earth image texture. Exercises spheres, motion blur, a spherical
// medium and checker textures.
void gen_cornell_spheres(mc_scene_host& s, std::vector<mc_triangle>& tris, std::vector<mc_sphere>& sph, uint64_t seed) {
    mc_material floor = base_material(MC_MAT_LAMBERTIAN);
    floor.albedo.type = MC_TEX_CHECKER;  // PT:211-213 make_checker_texture
    floor.albedo.color_a = srgb_to_linear(HV(0.9f, 0.9f, 0.9f));
    floor.albedo.color_b = srgb_to_linear(HV(0.1f, 0.1f, 0.1f));
    floor.albedo.scale = 8.f;
    mc_material white = make_lambertian(HV(0.73f, 0.73f, 0.73f));
    mc_material red = make_lambertian(HV(0.65f, 0.05f, 0.05f));
    mc_material green = make_lambertian(HV(0.12f, 0.45f, 0.15f));
    mc_material light = make_emissive(HV(15.0f, 15.0f, 15.0f));
    const float L = -2.f, R = 2.f, B = 0.f, T = 4.f, F = -4.f, N = 0.f;
    add_quad(tris, HV(L, B, N), HV(R, B, N), HV(R, B, F), HV(L, B, F), floor);
    add_quad(tris, HV(L, T, N), HV(R, T, N), HV(R, T, F), HV(L, T, F), white);
    add_quad(tris, HV(L, B, F), HV(R, B, F), HV(R, T, F), HV(L, T, F), white);
    add_quad(tris, HV(L, B, N), HV(L, B, F), HV(L, T, F), HV(L, T, N), red);
    add_quad(tris, HV(R, B, N), HV(R, B, F), HV(R, T, F), HV(R, T, N), green);
    add_quad(tris, HV(-1.f, T - 0.01f, -2.6f), HV(1.f, T - 0.01f, -2.6f), HV(1.f, T - 0.01f, -1.4f),
             HV(-1.f, T - 0.01f, -1.4f), light);
    HV boxCenter(-0.8f, 1.1f, -2.8f);
    add_box(tris, boxCenter, HV(0.55f, 1.1f, 0.55f), 0.3f, white);
    HV big(0.85f, 0.7f, -1.7f);
    sph.push_back(make_sphere(big, big, false, 0.7f, make_conductor(HV(0.9f, 0.9f, 0.9f), 0.02f)));
    HV smoke(0.f, 2.9f, -3.0f);
    sph.push_back(make_sphere(smoke, smoke, false, 0.6f, make_isotropic(HV(0.8f, 0.8f, 0.85f), 1.f)));
    SplitMix rng(seed ? seed : 42);
    const float r = 0.1f;
    for (int a = 0; a < 13; a++) {
        for (int b = 0; b < 13; b++) {
            float jx = ((float)rng.uniform() - 0.5f) * 0.08f, jz = ((float)rng.uniform() - 0.5f) * 0.08f;
            HV c(-1.8f + 0.3f * a + jx, r, -3.8f + 0.3f * b + jz);
            if ((c - big).length() < 0.7f + r + 0.02f) continue;
            if ((c - HV(boxCenter.x, r, boxCenter.z)).length() < 0.9f) continue;
            float choose = (float)rng.uniform();
            if (choose < 0.8f) {
                mc_material m = make_lambertian(HV((float)rng.uniform(), (float)rng.uniform(), (float)rng.uniform()));
                float h = 0.5f * (float)rng.uniform();
                sph.push_back(make_sphere(c, c + HV(0.f, h, 0.f), true, r, m));
            } else if (choose < 0.95f) {
                mc_material m = make_conductor(HV(0.5f + 0.5f * (float)rng.uniform(), 0.5f + 0.5f * (float)rng.uniform(),
                                                  0.5f + 0.5f * (float)rng.uniform()), 0.3f * (float)rng.uniform());
                sph.push_back(make_sphere(c, c, false, r, m));
            } else {
                sph.push_back(make_sphere(c, c, false, r, make_dielectric(1.5f)));
            }
        }
    }
    s.width = 512; s.height = 512; s.spp = 64; s.max_depth = 8;
    s.has_medium = 1;
    set_camera(s.camera, 512, 512, HV(0, 2, 5.5f), HV(0, 2, -2), 40.0f, 7.5f, 8, 64);
}

// Config: "displaced_icospheres" - three level-L icospheres (L = 8 by default:
// 1,310,720 triangles each) displaced radially by 0.05 * fbm4(value noise),
// randomly rotated, with per-instance materials from a seeded permutation of
// {diffuse, conductor fuzz~U[0,0.3], dielectric 1.5}, on a 2-triangle ground,
// a 12-triangle homogeneous isotropic box (density 0.5), a 2-triangle area
// light and a 2048x1024 procedural sky. 1920x1080, 16 spp, max depth 8.
void gen_icospheres(mc_scene_host& s, std::vector<mc_triangle>& tris, int level, uint64_t seed) {
    SplitMix rng(seed ? seed : 2);
    mc_material ground = make_lambertian(HV(0.5f, 0.5f, 0.5f));
    add_quad(tris, HV(-12, 0, 12), HV(12, 0, 12), HV(12, 0, -12), HV(-12, 0, -12), ground);
    int order[3] = {0, 1, 2};
    for (int i = 2; i > 0; i--) {
        int j = (int)(rng.next() % (uint64_t)(i + 1));
        std::swap(order[i], order[j]);
    }
    const double cx[3] = {-2.4, 0.0, 2.4}, cz[3] = {-0.5, 0.5, -0.5};
    for (int inst = 0; inst < 3; inst++) {
        mc_material m;
        float r0 = (float)rng.uniform(), r1 = (float)rng.uniform(), r2 = (float)rng.uniform(), r3 = (float)rng.uniform();
        switch (order[inst]) {
            case 0: m = make_lambertian(HV(0.3f + 0.6f * r0, 0.3f + 0.6f * r1, 0.3f + 0.6f * r2)); break;
            case 1: m = make_conductor(HV(0.6f + 0.35f * r0, 0.6f + 0.35f * r1, 0.6f + 0.35f * r2), 0.3f * r3); break;
            default: m = make_dielectric(1.5f); break;
        }
        Xform xf = random_rotation(rng);
        xf.t = DV{cx[inst], 1.05, cz[inst]};
        xf.scale = 1.0;
        Displace disp{0.05, 3.0, (uint32_t)(seed ? seed : 2) * 7919u + (uint32_t)inst};
        add_icosphere(tris, level, disp, xf, m);
    }
    mc_material fog = make_isotropic(HV(0.8f, 0.8f, 0.85f), 0.5f);
    add_box(tris, HV(0.f, 0.75f, 2.6f), HV(3.5f, 0.75f, 0.6f), 0.f, fog);
    mc_material light = make_emissive(HV(12.f, 12.f, 12.f));
    add_quad(tris, HV(-1, 6, -1), HV(1, 6, -1), HV(1, 6, 1), HV(-1, 6, 1), light);
    s.width = 1920; s.height = 1080; s.spp = 16; s.max_depth = 8;
    s.has_medium = 1;
    set_camera(s.camera, 1920, 1080, HV(0.f, 2.2f, 8.5f), HV(0.f, 1.0f, 0.f), 38.0f, 8.5f, 8, 16);
    std::vector<float> sky;
    make_sky(2048, 1024, sky);
    s.env_width = 2048;
    s.env_height = 1024;
    s.env_intensity = 1.0f;
    s.env_rgba = (float*)std::malloc(sky.size() * sizeof(float));
    std::memcpy(s.env_rgba, sky.data(), sky.size() * sizeof(float));
}

// Config: one of the 64 batch scenes. Triangle count log-normal (median 50k,
// sigma 1 in log space, clipped to [1k, 2M]); even members are displaced
// icospheres (instances of the largest level fitting the count), odd members
// random-triangle soups in [-1,1]^3 (centres uniform, corners within a cube of
// side 1.5 * N^(-1/3)). Resolution from {256^2, 512^2, 1024^2}, spp from {4, 16, 64}.
void gen_batch_member(mc_scene_host& s, std::vector<mc_triangle>& tris, int member, uint64_t seed, int target) {
    SplitMix rng((seed ? seed : 3) * 1000003ull + (uint64_t)member);
    double ln = std::log(50000.0) + rng.normal();
    long long count = target > 0 ? target : (long long)std::llround(std::exp(ln));
    count = std::max(1000ll, std::min(2000000ll, count));
    mc_material m = make_lambertian(HV(0.3f + 0.6f * (float)rng.uniform(), 0.3f + 0.6f * (float)rng.uniform(),
                                       0.3f + 0.6f * (float)rng.uniform()));
    if ((member & 1) == 0) {
        int level = 1;
        while (20ll * (1ll << (2 * (level + 1))) <= count && level < 8) level++;
        long long per = 20ll * (1ll << (2 * level));
        int instances = (int)std::max(1ll, (count + per / 2) / per);
        for (int i = 0; i < instances; i++) {
            Xform xf = random_rotation(rng);
            double sc = instances == 1 ? 0.9 : 0.9 / std::cbrt((double)instances);
            xf.t = DV{(rng.uniform() * 2 - 1) * (1 - sc), (rng.uniform() * 2 - 1) * (1 - sc), (rng.uniform() * 2 - 1) * (1 - sc)};
            xf.scale = sc;
            Displace disp{0.05, 3.0, (uint32_t)member * 31u + (uint32_t)i};
            add_icosphere(tris, level, disp, xf, m);
        }
    } else {
        double side = 1.5 * std::pow((double)count, -1.0 / 3.0);
        size_t base = tris.size();
        tris.resize(base + (size_t)count);
        for (long long i = 0; i < count; i++) {
            HV c((float)(rng.uniform() * 2 - 1), (float)(rng.uniform() * 2 - 1), (float)(rng.uniform() * 2 - 1));
            HV p[3];
            for (int k = 0; k < 3; k++)
                p[k] = c + HV((float)((rng.uniform() - 0.5) * side), (float)((rng.uniform() - 0.5) * side),
                              (float)((rng.uniform() - 0.5) * side));
            tris[base + (size_t)i] = make_triangle(p[0], p[1], p[2], m);
        }
    }
    mc_material light = make_emissive(HV(10.f, 10.f, 10.f));
    add_quad(tris, HV(-0.6f, 2.5f, -0.6f), HV(0.6f, 2.5f, -0.6f), HV(0.6f, 2.5f, 0.6f), HV(-0.6f, 2.5f, 0.6f), light);
    mc_material floor = make_lambertian(HV(0.6f, 0.6f, 0.6f));
    add_quad(tris, HV(-4, -1.2f, 4), HV(4, -1.2f, 4), HV(4, -1.2f, -4), HV(-4, -1.2f, -4), floor);
    const int res[3] = {256, 512, 1024}, spps[3] = {4, 16, 64};
    int r = res[rng.next() % 3];
    s.width = r; s.height = r;
    s.spp = spps[rng.next() % 3];
    s.max_depth = 8;
    set_camera(s.camera, r, r, HV(0.f, 0.8f, 3.6f), HV(0.f, 0.f, 0.f), 45.0f, 3.7f, 8, s.spp);
}

// Config: "guiding_room" - a 10x10x4 closed room (floor, walls, ceiling with a
// 0.2x0.2 opening at its centre) furnished with random boxes and level-5/6
// displaced spheres (about 200k triangles), lit only by a 500-radiance quad
// above the opening. 1024x1024.
void gen_guiding_room(mc_scene_host& s, std::vector<mc_triangle>& tris, uint64_t seed) {
    SplitMix rng(seed ? seed : 4);
    mc_material wall = make_lambertian(HV(0.75f, 0.75f, 0.75f));
    const float X = 5.f, Z = 5.f, Y = 4.f, a = 0.1f;
    add_quad(tris, HV(-X, 0, Z), HV(X, 0, Z), HV(X, 0, -Z), HV(-X, 0, -Z), wall);       // floor
    add_quad(tris, HV(-X, 0, -Z), HV(X, 0, -Z), HV(X, Y, -Z), HV(-X, Y, -Z), wall);     // back
    add_quad(tris, HV(-X, 0, Z), HV(-X, Y, Z), HV(X, Y, Z), HV(X, 0, Z), wall);         // front
    add_quad(tris, HV(-X, 0, Z), HV(-X, 0, -Z), HV(-X, Y, -Z), HV(-X, Y, Z), wall);     // left
    add_quad(tris, HV(X, 0, -Z), HV(X, 0, Z), HV(X, Y, Z), HV(X, Y, -Z), wall);         // right
    // ceiling with a square hole [-a, a]^2: four quads around it
    add_quad(tris, HV(-X, Y, -Z), HV(X, Y, -Z), HV(X, Y, -a), HV(-X, Y, -a), wall);
    add_quad(tris, HV(-X, Y, a), HV(X, Y, a), HV(X, Y, Z), HV(-X, Y, Z), wall);
    add_quad(tris, HV(-X, Y, -a), HV(-a, Y, -a), HV(-a, Y, a), HV(-X, Y, a), wall);
    add_quad(tris, HV(a, Y, -a), HV(X, Y, -a), HV(X, Y, a), HV(a, Y, a), wall);
    mc_material light = make_emissive(HV(500.f, 500.f, 500.f));
    add_quad(tris, HV(-0.3f, Y + 0.5f, -0.3f), HV(-0.3f, Y + 0.5f, 0.3f), HV(0.3f, Y + 0.5f, 0.3f),
             HV(0.3f, Y + 0.5f, -0.3f), light);
    for (int b = 0; b < 40; b++) {
        HV half((float)(0.2 + 0.5 * rng.uniform()), (float)(0.1 + 0.6 * rng.uniform()), (float)(0.2 + 0.5 * rng.uniform()));
        HV c((float)((rng.uniform() * 2 - 1) * 4.0), half.y, (float)((rng.uniform() * 2 - 1) * 4.0));
        add_box(tris, c, half, (float)(rng.uniform() * M_PI), make_lambertian(HV(0.4f + 0.5f * (float)rng.uniform(), 0.4f + 0.5f * (float)rng.uniform(), 0.4f + 0.5f * (float)rng.uniform())));
    }
    const int levels[4] = {6, 6, 5, 5};
    for (int i = 0; i < 4; i++) {
        Xform xf = random_rotation(rng);
        double r = 0.4 + 0.3 * rng.uniform();
        xf.t = DV{(rng.uniform() * 2 - 1) * 3.5, r, (rng.uniform() * 2 - 1) * 3.5};
        xf.scale = r;
        Displace disp{0.05, 3.0, 4000u + (uint32_t)i};
        add_icosphere(tris, levels[i], disp, xf, make_lambertian(HV(0.7f, 0.7f, 0.7f)));
    }
    s.width = 1024; s.height = 1024; s.spp = 16; s.max_depth = 8;
    set_camera(s.camera, 1024, 1024, HV(0.f, 2.0f, 4.8f), HV(0.f, 1.2f, 0.f), 70.0f, 5.0f, 8, 16);
}


const char* generate(const mc_scene_desc* desc, mc_scene_host* out, mc_status* status) {
    *status = MC_ERR_INVALID;
    if (out) std::memset(out, 0, sizeof(*out));
    if (!desc || !out) return "mc_scene_generate: null argument";
    std::vector<mc_triangle> tris;
    std::vector<mc_sphere> sph;
    switch (desc->kind) {
        case MC_SCENE_CORNELL_BOXES: gen_cornell_boxes(*out, tris); break;
        case MC_SCENE_CORNELL_SPHERES: gen_cornell_spheres(*out, tris, sph, desc->seed); break;
        case MC_SCENE_DISPLACED_ICOSPHERES: {
            int level = desc->variant > 0 ? desc->variant : 8;
            if (level > 9) return "mc_scene_generate: icosphere level must be <= 9";
            gen_icospheres(*out, tris, level, desc->seed);
            break;
        }
        case MC_SCENE_BATCH_MEMBER:
            if (desc->variant < 0) return "mc_scene_generate: bad batch member";
            gen_batch_member(*out, tris, desc->variant, desc->seed, desc->triangle_target);
            break;
        case MC_SCENE_GUIDING_ROOM: gen_guiding_room(*out, tris, desc->seed); break;
        default: return "mc_scene_generate: unknown scene kind";
    }
    finalize(tris.data(), (int32_t)tris.size(), nullptr, nullptr);
    out->triangle_count = (int32_t)tris.size();
    out->triangles = (mc_triangle*)std::malloc(sizeof(mc_triangle) * (tris.empty() ? 1 : tris.size()));
    if (!out->triangles) { *status = MC_ERR_OOM; return "mc_scene_generate: host allocation failed"; }
    if (!tris.empty()) std::memcpy(out->triangles, tris.data(), sizeof(mc_triangle) * tris.size());
    out->sphere_count = (int32_t)sph.size();
    out->spheres = nullptr;
    if (!sph.empty()) {
        out->spheres = (mc_sphere*)std::malloc(sizeof(mc_sphere) * sph.size());
        if (!out->spheres) { *status = MC_ERR_OOM; return "mc_scene_generate: host allocation failed"; }
        std::memcpy(out->spheres, sph.data(), sizeof(mc_sphere) * sph.size());
    }
    *status = MC_OK;
    return nullptr;
}


void free_scene(mc_scene_host* s) {
    if (!s) return;
    std::free(s->triangles);
    std::free(s->spheres);
    std::free(s->env_rgba);
    std::memset(s, 0, sizeof(*s));
}

}  // namespace mc_gen
