// mc_host_scene.h - host-side scene helpers shared by the scene generators and
// the OBJ loader: the reference's host vec3 arithmetic (operations in the
// reference's order; the including files are compiled with -ffp-contract=off)
// and its material and texture constructors (PT:201-209, 581-603).
#pragma once
#include <cmath>
#include <cstring>

#include "mc_abi.h"

namespace mc_host {

struct HV {
    float x, y, z;
    HV() : x(0), y(0), z(0) {}
    HV(float a, float b, float c) : x(a), y(b), z(c) {}
    HV(const mc_vec3& v) : x(v.x), y(v.y), z(v.z) {}
    operator mc_vec3() const { return mc_vec3{x, y, z}; }
    HV operator+(const HV& o) const { return HV(x + o.x, y + o.y, z + o.z); }
    HV operator-(const HV& o) const { return HV(x - o.x, y - o.y, z - o.z); }
    HV operator-() const { return HV(-x, -y, -z); }
    HV operator*(float s) const { return HV(x * s, y * s, z * s); }
    HV operator/(float s) const { return HV(x / s, y / s, z / s); }
    float length_squared() const { return x * x + y * y + z * z; }
    float length() const { return std::sqrt(length_squared()); }
    HV cross(const HV& o) const { return HV(y * o.z - z * o.y, z * o.x - x * o.z, x * o.y - y * o.x); }
    float dot(const HV& o) const { return x * o.x + y * o.y + z * o.z; }
    HV normalize() const {
        float len = std::sqrt(length_squared());
        return HV(x / len, y / len, z / len);
    }
};

// PT:201-206 srgbToLinear (host evaluation, as make_solid_texture runs on the host)
inline float srgb_to_linear(float c) { return c <= 0.04045f ? c / 12.92f : powf((c + 0.055f) / 1.055f, 2.4f); }
inline HV srgb_to_linear(const HV& c) { return HV(srgb_to_linear(c.x), srgb_to_linear(c.y), srgb_to_linear(c.z)); }

inline mc_texture solid_texture(HV color) {  // PT:207-209 make_solid_texture
    mc_texture t;
    std::memset(&t, 0, sizeof(t));
    t.type = MC_TEX_SOLID;
    t.color_a = srgb_to_linear(color);
    t.color_b = mc_vec3{0, 0, 0};
    t.scale = 1.f;
    t.image = 0;
    return t;
}

inline mc_material base_material(int type) {
    mc_material m;
    std::memset(&m, 0, sizeof(m));
    m.type = type;
    return m;
}

// PT:581-603 material constructors
inline mc_material make_lambertian(HV albedo) {
    mc_material m = base_material(MC_MAT_LAMBERTIAN);
    m.albedo = solid_texture(albedo);
    return m;
}
inline mc_material make_conductor(HV albedo, float fuzz) {
    mc_material m = base_material(MC_MAT_CONDUCTOR);
    m.albedo = solid_texture(albedo);
    m.fuzz = fuzz < 1 ? fuzz : 1.f;
    return m;
}
inline mc_material make_dielectric(float ior) {
    mc_material m = base_material(MC_MAT_DIELECTRIC);
    m.albedo = solid_texture(HV(1, 1, 1));
    m.refraction_index = ior;
    return m;
}
inline mc_material make_emissive(HV color) {
    mc_material m = base_material(MC_MAT_EMISSIVE);
    m.albedo = solid_texture(HV(0, 0, 0));
    m.emitted = color;
    return m;
}
inline mc_material make_isotropic(HV albedo, float density, float g = 0.f) {
    mc_material m = base_material(MC_MAT_ISOTROPIC);
    m.albedo = solid_texture(albedo);
    m.density = density;
    m.phase_g = g;
    return m;
}

inline mc_triangle make_triangle(HV a, HV b, HV c, const mc_material& m) {
    mc_triangle t;
    std::memset(&t, 0, sizeof(t));
    t.v0 = a;
    t.v1 = b;
    t.v2 = c;
    t.mat = m;
    return t;
}

}  // namespace mc_host
