// mc_scene_gen.h - the seeded synthetic scenes (mc_scene_gen.cpp) and the host
// scene helpers they are built from. Host-only; no dependency on the rest of
// the library.
#pragma once
#include <cstdint>
#include <vector>

#include "mc_abi.h"
#include "mc_host_scene.h"

namespace mc_gen {

// PT:1610-1631 Camera::initialize (look_from, look_at, up, vfov, aperture,
// focus distance, image width and aspect ratio set).
void camera_initialize(mc_camera& cam);
// PT:651-655 triangle bounds and PT:1972-1985 emissive-triangle light list
// (lights may be null to count only).
void finalize(mc_triangle* tris, int32_t n, mc_light* lights, int32_t* light_count);
// PT:1677-1691 add_quad, PT:1693-1708 add_box.
void add_quad(std::vector<mc_triangle>& tris, mc_host::HV a, mc_host::HV b, mc_host::HV c, mc_host::HV d,
              const mc_material& m);
void add_box(std::vector<mc_triangle>& tris, mc_host::HV center, mc_host::HV half, float rotY, const mc_material& m);
// A sphere with its bounding box (PT:850-859).
mc_sphere make_sphere(mc_host::HV c0, mc_host::HV c1, bool moving, float r, const mc_material& m);
// A pinhole camera of the given film, view and depth, initialized.
void set_camera(mc_camera& cam, int W, int H, mc_host::HV from, mc_host::HV at, float vfov, float focus, int depth,
                int spp);
// Generates desc's scene into out (host arrays from malloc, released by
// free_scene). Returns null on success, else a message, with the status in *status.
const char* generate(const mc_scene_desc* desc, mc_scene_host* out, mc_status* status);
void free_scene(mc_scene_host* s);

}  // namespace mc_gen
