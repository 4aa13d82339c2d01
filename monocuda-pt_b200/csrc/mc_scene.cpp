// mc_scene.cpp - host side of the scene surface behind the C ABI: camera
// set-up, scene finalization (bounds, light list), the hot/cold split, the
// cloud scene, the seeded synthetic scenes (generated by mc_scene_gen.cpp) and
// the environment-map sampling tables.
//
// Compiled by the host compiler with -ffp-contract=off: the reference runs the
// same steps on the host (Camera::initialize PT:1610-1631, finalizeScene
// PT:1930-1987, buildEnvironmentSamplingTables PT:370-385), so the float
// results are bit-identical when the operations are written in the same order.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "mc_abi.h"
#include "mc_host_scene.h"
#include "mc_internal.h"
#include "mc_scene_gen.h"

using namespace mc_host;
using mc_gen::add_quad;
using mc_gen::make_sphere;
using mc_gen::set_camera;

extern "C" {

mc_status mc_camera_initialize(mc_camera* cam) {
    if (!cam) return mc::set_error(MC_ERR_INVALID, "mc_camera_initialize: null camera");
    mc_gen::camera_initialize(*cam);
    return MC_OK;
}

mc_status mc_scene_finalize_host(mc_triangle* tris, int32_t n, mc_light* lights, int32_t* light_count) {
    if (n < 0 || (n > 0 && !tris)) return mc::set_error(MC_ERR_INVALID, "mc_scene_finalize_host: bad triangles");
    mc_gen::finalize(tris, n, lights, light_count);
    return MC_OK;
}

// PT:4276-4281 hot/cold split.
mc_status mc_split_triangles_host(const mc_triangle* tris, int32_t n, mc_triangle_hot* hot, mc_triangle_cold* cold) {
    if (n < 0 || (n > 0 && (!tris || !hot || !cold))) return mc::set_error(MC_ERR_INVALID, "mc_split_triangles_host: bad arguments");
    for (int32_t i = 0; i < n; i++) {
        const mc_triangle& t = tris[i];
        hot[i].v0 = t.v0; hot[i].v1 = t.v1; hot[i].v2 = t.v2;
        cold[i].uv0 = t.uv0; cold[i].uv1 = t.uv1; cold[i].uv2 = t.uv2;
        cold[i].n0 = t.n0; cold[i].n1 = t.n1; cold[i].n2 = t.n2;
        cold[i].mat = t.mat;
        cold[i].aabb = t.aabb;
    }
    return MC_OK;
}

mc_status mc_scene_cloud(const mc_volume_grid* d_grid, const mc_volume_grid* header, int32_t sun, mc_scene_host* out) {
    if (!d_grid || !header || !out) return mc::set_error(MC_ERR_INVALID, "mc_scene_cloud: null argument");
    std::memset(out, 0, sizeof(*out));
    const HV gmin(header->world_min[0], header->world_min[1], header->world_min[2]);
    const HV gmax(header->world_max[0], header->world_max[1], header->world_max[2]);
    const HV center = (gmin + gmax) * 0.5f;
    const float radius = (gmax - gmin).length() * 0.5f;
    if (!(radius > 0.f)) return mc::set_error(MC_ERR_INVALID, "mc_scene_cloud: the grid has no extent");
    std::vector<mc_triangle> tris;
    std::vector<mc_sphere> sph;
    // PT:1863-1866: an isotropic sphere around the grid (density scale 4,
    // Henyey-Greenstein g 0.877, PT:1721-1722); the grid goes into every
    // medium's material as main() does (PT:2509-2520)
    mc_material cloud = make_isotropic(HV(1.f, 1.f, 1.f), 4.0f, 0.877f);
    cloud.density_grid = d_grid;
    cloud.grid_max_density = header->maximum_density;
    sph.push_back(make_sphere(center, center, false, radius, cloud));
    sph.back().center1 = mc_vec3{0.f, 0.f, 0.f};  // a stationary sphere's unused second centre, as the reference leaves it
    // PT:1868-1872: the ground that lights the cloud's underside
    const float extent = 20000.f, height = -1000.f;
    add_quad(tris, HV(-extent, height, -extent), HV(extent, height, -extent), HV(extent, height, extent),
             HV(-extent, height, extent), make_lambertian(HV(0.2f, 0.2f, 0.2f)));
    if (sun) {
        // PT:1874-1891: the directional sun as a far quad of matching irradiance
        // (E = L * area / distance^2)
        const HV toSun = -HV(-0.5826f, -0.7660f, -0.2717f);
        const float distance = 8.f * radius;
        const float half = 0.1f * distance;
        const float scale = (distance * distance) / (4.f * half * half);
        const mc_material light = make_emissive(HV(2.6f, 2.5f, 2.3f) * scale);
        const HV c = center + toSun * distance;
        const HV helper = (std::fabs(toSun.x) > 0.9f) ? HV(0.f, 1.f, 0.f) : HV(1.f, 0.f, 0.f);
        const HV tangent = helper.cross(toSun).normalize() * half;
        const HV bitangent = toSun.cross(tangent.normalize()) * half;
        add_quad(tris, c - tangent - bitangent, c + tangent - bitangent, c + tangent + bitangent, c - tangent + bitangent,
                 light);
    }
    // main()'s film and camera for the cloud (PT:4080-4084, 4113-4126, 4148-4167):
    // the Mitsuba sensor, its horizontal field of view turned vertical, deep paths
    const int W = 333, H = 180;
    const float pi = 3.14159265358979323846f;
    const float hfov = 54.43f * pi / 180.f;
    const float aspect = (float)W / (float)H;
    const HV from(648.064f, -82.473f, -63.856f), at(6.021f, 100.043f, -43.679f);
    set_camera(out->camera, W, H, from, at, 2.f * std::atan(std::tan(hfov * 0.5f) / aspect) * 180.f / pi,
               (at - from).length(), 1000, 500);
    out->camera.up = mc_vec3{0.273f, 0.962f, -0.009f};
    out->camera.background = mc_vec3{0.03f, 0.07f, 0.23f};
    out->camera.rr_cap = 0.95f;
    mc_camera_initialize(&out->camera);
    out->width = W;
    out->height = H;
    out->spp = 500;
    out->max_depth = 1000;
    out->has_medium = MC_MEDIUM_ANY | MC_MEDIUM_GRID;
    mc_scene_finalize_host(tris.data(), (int32_t)tris.size(), nullptr, nullptr);
    out->triangle_count = (int32_t)tris.size();
    out->triangles = (mc_triangle*)std::malloc(sizeof(mc_triangle) * tris.size());
    out->sphere_count = (int32_t)sph.size();
    out->spheres = (mc_sphere*)std::malloc(sizeof(mc_sphere) * sph.size());
    if (!out->triangles || !out->spheres) {
        mc_scene_free(out);
        return mc::set_error(MC_ERR_OOM, "mc_scene_cloud: host allocation failed");
    }
    std::memcpy(out->triangles, tris.data(), sizeof(mc_triangle) * tris.size());
    std::memcpy(out->spheres, sph.data(), sizeof(mc_sphere) * sph.size());
    return MC_OK;
}

mc_status mc_scene_generate(const mc_scene_desc* desc, mc_scene_host* out) {
    mc_status st = MC_OK;
    const char* msg = mc_gen::generate(desc, out, &st);
    if (msg) {
        if (out) mc_gen::free_scene(out);
        return mc::set_error(st, "%s", msg);
    }
    return MC_OK;
}

mc_status mc_scene_free(mc_scene_host* s) {
    mc_gen::free_scene(s);
    return MC_OK;
}

}  // extern "C"

namespace mc {

// PT:370-385 buildEnvironmentSamplingTables, same accumulation order.
void build_env_tables(const float* rgba, int W, int H, std::vector<float>& rowCdf, std::vector<float>& colCdf, float& total) {
    rowCdf.assign((size_t)H + 1, 0.0f);
    colCdf.assign((size_t)H * (W + 1), 0.0f);
    for (int row = 0; row < H; row++) {
        float sinTheta = sinf(3.14159265358979323846f * (row + 0.5f) / H);
        float* cdf = &colCdf[(size_t)row * (W + 1)];
        cdf[0] = 0.0f;
        for (int col = 0; col < W; col++) {
            const float* t = &rgba[((size_t)row * W + col) * 4];
            float lum = 0.2126f * t[0] + 0.7152f * t[1] + 0.0722f * t[2];
            cdf[col + 1] = cdf[col] + fmaxf(lum, 0.0f) * sinTheta;
        }
        rowCdf[row + 1] = rowCdf[row] + cdf[W];
    }
    total = rowCdf[H];
}

}  // namespace mc
