// monocuda - command-line driver over the C ABI.
//
// Mirrors the reference executable's render flags (parseCommandLine,
// src/path_tracer.cu:3908-3964): --wavefront, --persistent, --scene NAME,
// --spp N, plus the settings the reference fixes in main() (resolution
// PT:4080-4081, max depth PT:4117, seed PT:4297) and this library's own
// choices (RNG, intersector, CUDA graph). The scenes are the
// library's seeded generators. --tonemap and --exposure follow the reference's
// flags; the image is resolved once after the last sample (mc_image_encode)
// and written by the extension of --out: .png (the reference's output: tone
// mapped, sRGB, 8-bit), .ppm (the same pixels), .pfm (linear radiance times
// the exposure). --env / --env-intensity / --env-rotation load a PFM
// environment map as the reference does (PT:4186-4221; its EXR/HDR readers
// belong to image libraries this build does not include), --phase-g sets the
// Henyey-Greenstein g of every medium (PT:4059, 2505-2508) and --volume fills
// every medium with a dense density grid file (the reference's .nvdb grid,
// PT:4066-4076, 2509-2520; see mc_volume_file_read). --pbrt and
// --max-triangles (pbrt scene import) are refused.
//
// Exit status: 0 on success, 1 on a library error (message on stderr), 2 on a
// usage error.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "mc_abi.h"

namespace {

struct Options {
    bool wavefront = false;
    bool persistent = false;
    std::string scene = "cornell_boxes";
    int variant = 0;
    uint64_t sceneSeed = 0;
    int spp = 0;
    int width = 0;
    int height = 0;
    int maxDepth = 0;
    uint64_t seed = 1234;
    int rng = MC_RNG_PHILOX;
    int intersector = MC_ISECT_REFERENCE;
    bool graph = false;
    std::string out;
    bool stats = false;
    int tonemap = MC_TONEMAP_NONE;
    float exposure = 1.0f;  // <= 0: automatic
    std::string envPath;
    float envIntensity = 1.0f;
    bool envIntensitySet = false;
    float envRotationDegrees = 0.0f;
    float phaseG = 0.0f;
    bool phaseGSet = false;
    std::string volumePath;
};

constexpr float kPi = 3.14159265358979323846f;

const struct {
    const char* name;
    int kind;
} kScenes[] = {{"cornell_boxes", MC_SCENE_CORNELL_BOXES},
               {"cornell_spheres", MC_SCENE_CORNELL_SPHERES},
               {"displaced_icospheres", MC_SCENE_DISPLACED_ICOSPHERES},
               {"guiding_room", MC_SCENE_GUIDING_ROOM},
               {"batch_member", MC_SCENE_BATCH_MEMBER}};

void usage(FILE* f) {
    std::fprintf(f,
                 "usage: monocuda [--wavefront] [--persistent] [--scene NAME] [--spp N]\n"
                 "                [--width W] [--height H] [--depth D] [--seed S] [--variant V] [--scene-seed S]\n"
                 "                [--rng philox|xorwow] [--watertight] [--graph]\n"
                 "                [--tonemap none|reinhard|aces] [--exposure X|auto]\n"
                 "                [--out FILE.png|FILE.ppm|FILE.pfm] [--stats]\n"
                 "                [--env FILE.pfm] [--env-intensity X] [--env-rotation DEGREES] [--phase-g G]\n"
                 "                [--volume FILE]\n"
                 "scenes:");
    for (const auto& s : kScenes) std::fprintf(f, " %s", s.name);
    std::fprintf(f, " cloud (with --volume)\n");
}

bool parse(int argc, char** argv, Options& o) {
    for (int i = 1; i < argc; i++) {
        const char* a = argv[i];
        auto next = [&](const char* flag) -> const char* {
            if (i + 1 >= argc) {
                std::fprintf(stderr, "%s needs a value\n", flag);
                return nullptr;
            }
            return argv[++i];
        };
        const char* v = nullptr;
        if (!std::strcmp(a, "--wavefront")) o.wavefront = true;
        else if (!std::strcmp(a, "--persistent")) o.persistent = true;
        else if (!std::strcmp(a, "--watertight")) o.intersector = MC_ISECT_WATERTIGHT;
        else if (!std::strcmp(a, "--graph")) o.graph = true;
        else if (!std::strcmp(a, "--stats")) o.stats = true;
        else if (!std::strcmp(a, "--help") || !std::strcmp(a, "-h")) {
            usage(stdout);
            std::exit(0);
        } else if (!std::strcmp(a, "--scene")) {
            if (!(v = next(a))) return false;
            o.scene = v;
        } else if (!std::strcmp(a, "--spp")) {
            if (!(v = next(a))) return false;
            o.spp = std::atoi(v);
        } else if (!std::strcmp(a, "--width")) {
            if (!(v = next(a))) return false;
            o.width = std::atoi(v);
        } else if (!std::strcmp(a, "--height")) {
            if (!(v = next(a))) return false;
            o.height = std::atoi(v);
        } else if (!std::strcmp(a, "--depth")) {
            if (!(v = next(a))) return false;
            o.maxDepth = std::atoi(v);
        } else if (!std::strcmp(a, "--seed")) {
            if (!(v = next(a))) return false;
            o.seed = std::strtoull(v, nullptr, 10);
        } else if (!std::strcmp(a, "--scene-seed")) {
            if (!(v = next(a))) return false;
            o.sceneSeed = std::strtoull(v, nullptr, 10);
        } else if (!std::strcmp(a, "--variant")) {
            if (!(v = next(a))) return false;
            o.variant = std::atoi(v);
        } else if (!std::strcmp(a, "--rng")) {
            if (!(v = next(a))) return false;
            if (!std::strcmp(v, "philox")) o.rng = MC_RNG_PHILOX;
            else if (!std::strcmp(v, "xorwow")) o.rng = MC_RNG_XORWOW;
            else {
                std::fprintf(stderr, "unknown rng '%s'\n", v);
                return false;
            }
        } else if (!std::strcmp(a, "--tonemap")) {
            // PT:3933-3936: unknown names leave the default (none)
            if (!(v = next(a))) return false;
            if (!std::strcmp(v, "reinhard")) o.tonemap = MC_TONEMAP_REINHARD;
            else if (!std::strcmp(v, "aces")) o.tonemap = MC_TONEMAP_ACES;
        } else if (!std::strcmp(a, "--exposure")) {
            // PT:3937-3944: "auto", or a positive multiplier (others are ignored)
            if (!(v = next(a))) return false;
            if (!std::strcmp(v, "auto")) o.exposure = 0.0f;
            else if ((float)std::atof(v) > 0.0f) o.exposure = (float)std::atof(v);
        } else if (!std::strcmp(a, "--out")) {
            if (!(v = next(a))) return false;
            o.out = v;
        } else if (!std::strcmp(a, "--env")) {
            if (!(v = next(a))) return false;
            o.envPath = v;
        } else if (!std::strcmp(a, "--env-intensity")) {
            if (!(v = next(a))) return false;
            o.envIntensity = (float)std::atof(v);
            o.envIntensitySet = true;
        } else if (!std::strcmp(a, "--env-rotation")) {
            if (!(v = next(a))) return false;
            o.envRotationDegrees = (float)std::atof(v);
        } else if (!std::strcmp(a, "--phase-g")) {
            if (!(v = next(a))) return false;
            o.phaseG = (float)std::atof(v);
            o.phaseGSet = true;
        } else if (!std::strcmp(a, "--volume")) {
            if (!(v = next(a))) return false;
            o.volumePath = v;
        } else if (!std::strcmp(a, "--pbrt") || !std::strcmp(a, "--max-triangles")) {
            std::fprintf(stderr, "%s: pbrt scene import is not part of this build\n", a);
            return false;
        } else {
            std::fprintf(stderr, "unknown argument '%s'\n", a);
            return false;
        }
    }
    if (o.persistent && !o.wavefront) {
        // as the reference (PT:4051-4053): --persistent alone is ignored
        std::printf("--persistent only applies to the wavefront path tracer, ignoring it (add --wavefront)\n");
        o.persistent = false;
    }
    return true;
}

int fail(const char* what, mc_status s) {
    std::fprintf(stderr, "%s: %s: %s\n", what, mc_status_string(s), mc_last_error());
    return 1;
}

bool ends_with(const std::string& s, const char* suffix) {
    const size_t n = std::strlen(suffix);
    return s.size() >= n && s.compare(s.size() - n, n, suffix) == 0;
}

bool write_file(const std::string& path, const void* head, size_t headBytes, const void* data, size_t bytes) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    bool ok = std::fwrite(head, 1, headBytes, f) == headBytes && std::fwrite(data, 1, bytes, f) == bytes;
    return (std::fclose(f) == 0) && ok;
}

}  // namespace

int main(int argc, char** argv) {
    Options o;
    if (!parse(argc, argv, o)) {
        usage(stderr);
        return 2;
    }
    int kind = 0;
    for (const auto& s : kScenes)
        if (o.scene == s.name) kind = s.kind;
    if (!kind && o.scene != "cloud") {
        std::fprintf(stderr, "unknown scene '%s'\n", o.scene.c_str());
        usage(stderr);
        return 2;
    }
    if (!o.wavefront)
        std::fprintf(stderr, "note: this library has only the wavefront path; rendering with it (the megakernel is not part of it)\n");
    // the environment map and the grid are read before any device work
    std::vector<float> envPixels;
    int envW = 0, envH = 0;
    if (!o.envPath.empty()) {
        mc_status es = MC_OK;
        if (!ends_with(o.envPath, ".pfm")) {
            std::fprintf(stderr, "could not load environment map '%s': only PFM files are read (EXR and HDR need image "
                                 "libraries this build does not include)\n", o.envPath.c_str());
            return 1;
        }
        if ((es = mc_pfm_read(o.envPath.c_str(), &envW, &envH, nullptr)) == MC_OK) {
            envPixels.resize((size_t)envW * envH * 4);
            es = mc_pfm_read(o.envPath.c_str(), &envW, &envH, envPixels.data());
        }
        if (es != MC_OK) return fail("could not load environment map", es);
    }
    std::vector<float> density;
    int32_t gridDims[3] = {0, 0, 0};
    float gridOrigin[3] = {0, 0, 0}, voxel = 0.f;
    if (!o.volumePath.empty()) {
        mc_status vs = mc_volume_file_read(o.volumePath.c_str(), gridDims, gridOrigin, &voxel, nullptr);
        if (vs == MC_OK) {
            density.resize((size_t)gridDims[0] * gridDims[1] * gridDims[2]);
            vs = mc_volume_file_read(o.volumePath.c_str(), gridDims, gridOrigin, &voxel, density.data());
        }
        if (vs != MC_OK) return fail("could not load volume", vs);
    }

    // the cloud scene is built around the grid (buildCloudScene, PT:1849-1891)
    const bool cloud = o.scene == "cloud";
    if (cloud && density.empty()) {
        std::fprintf(stderr, "the cloud scene needs a density grid: pass one with --volume FILE\n");
        return 1;
    }
    mc_status st = MC_OK;
    mc_context* ctx = nullptr;
    if ((st = mc_context_create(0, &ctx)) != MC_OK) return fail("mc_context_create", st);
    const mc_volume_grid* grid = nullptr;
    mc_volume_grid header = {};
    mc_scene_host scene = {};
    mc_env_map env = {};
    auto cleanup = [&]() {
        mc_env_destroy(&env);
        mc_volume_grid_destroy(grid);
        mc_context_destroy(ctx);
        mc_scene_free(&scene);
    };
    if (!density.empty() &&
        (st = mc_volume_grid_create(ctx, density.data(), gridDims[0], gridDims[1], gridDims[2], gridOrigin, voxel, &grid,
                                    &header)) != MC_OK) {
        cleanup();
        return fail("mc_volume_grid_create", st);
    }
    if (cloud) {
        st = mc_scene_cloud(grid, &header, envPixels.empty() ? 1 : 0, &scene);  // the sun quad without --env
    } else {
        mc_scene_desc desc = {};
        desc.kind = kind;
        desc.variant = o.variant;
        desc.seed = o.sceneSeed;
        st = mc_scene_generate(&desc, &scene);
    }
    if (st != MC_OK) {
        cleanup();
        return fail(cloud ? "mc_scene_cloud" : "mc_scene_generate", st);
    }
    auto forEachMedium = [&](auto&& fn) {
        int n = 0;
        for (int i = 0; i < scene.sphere_count; i++)
            if (scene.spheres[i].mat.type == MC_MAT_ISOTROPIC) fn(scene.spheres[i].mat), n++;
        for (int i = 0; i < scene.triangle_count; i++)
            if (scene.triangles[i].mat.type == MC_MAT_ISOTROPIC) fn(scene.triangles[i].mat), n++;
        return n;
    };
    if (o.phaseGSet) {
        const float g = std::fmin(std::fmax(o.phaseG, -0.99f), 0.99f);
        forEachMedium([&](mc_material& m) { m.phase_g = g; });
    }
    if (grid) {
        // every medium takes the grid (PT:2509-2520)
        const int media = forEachMedium([&](mc_material& m) {
            m.density_grid = grid;
            m.grid_max_density = header.maximum_density;
        });
        std::printf("volume '%s': %dx%dx%d voxels, maximum density %.3f, %d medium primitives\n", o.volumePath.c_str(),
                    gridDims[0], gridDims[1], gridDims[2], header.maximum_density, media);
    }

    const int W = o.width > 0 ? o.width : scene.width;
    const int H = o.height > 0 ? o.height : (o.width > 0 ? (int)((long long)scene.height * W / scene.width) : scene.height);
    mc_camera cam = scene.camera;
    if (W != scene.width || H != scene.height) {
        cam.image_width = W;
        cam.aspect_ratio = (float)W / (float)H;
        if ((st = mc_camera_initialize(&cam)) != MC_OK) {
            cleanup();
            return fail("mc_camera_initialize", st);
        }
    }
    const float envRotation = o.envRotationDegrees * kPi / 180.0f;  // PT:4193
    if (!envPixels.empty()) {
        st = mc_env_create(envPixels.data(), envW, envH, o.envIntensity, envRotation, &env);
        if (st == MC_OK)
            std::printf("Environment map: %s (%dx%d), intensity %g, rotation %g deg\n", o.envPath.c_str(), envW, envH,
                        o.envIntensity, o.envRotationDegrees);
    } else if (scene.env_rgba) {
        st = mc_env_create(scene.env_rgba, scene.env_width, scene.env_height,
                           o.envIntensitySet ? o.envIntensity : scene.env_intensity, envRotation, &env);
    }
    if (st != MC_OK) {
        cleanup();
        return fail("mc_env_create", st);
    }

    mc_render_params p = {};
    p.camera = cam;
    p.width = W;
    p.height = H;
    p.spp = o.spp > 0 ? o.spp : scene.spp;
    p.max_depth = o.maxDepth > 0 ? o.maxDepth : scene.max_depth;
    p.persistent = o.persistent ? 1 : 0;
    p.rng = o.rng;
    p.seed = o.seed;
    p.intersector = o.intersector;
    p.use_graph = o.graph ? 1 : 0;
    p.refill_threshold = 0;

    std::vector<float> accum((size_t)W * H * 3, 0.f);
    mc_render_stats stats = {};
    st = mc_render_host(ctx, scene.triangles, scene.triangle_count, scene.spheres, scene.sphere_count, &env, &p,
                        accum.data(), &stats);
    int rc = 0;
    if (st != MC_OK) {
        rc = fail("mc_render_host", st);
    } else {
        long long rays = stats.extend_rays + stats.shadow_rays;
        std::printf("%s: %dx%d, %d spp, depth %d, %d triangles, %d spheres\n", o.scene.c_str(), W, H, p.spp, p.max_depth,
                    scene.triangle_count, scene.sphere_count);
        std::printf("render %.3f ms, %lld rays, %.1f Mrays/s\n", stats.render_ms, rays,
                    stats.render_ms > 0 ? rays / (stats.render_ms * 1e3) : 0.0);
        if (o.stats) {
            for (int d = 0; d < MC_MAX_DEPTH_STATS && (stats.extend_per_depth[d] || stats.shadow_per_depth[d]); d++)
                std::printf("  bounce %d: %lld extend, %lld shadow\n", d, (long long)stats.extend_per_depth[d],
                            (long long)stats.shadow_per_depth[d]);
        }
        if (!o.out.empty()) {
            mc_image_options io = {};
            io.format = ends_with(o.out, ".pfm") ? MC_IMAGE_PFM : ends_with(o.out, ".png") ? MC_IMAGE_PNG : MC_IMAGE_RGB8;
            io.tonemap = o.tonemap;
            io.exposure = o.exposure;
            int64_t bytes = 0;
            float chosen = 0.f;
            std::vector<uint8_t> img;
            st = mc_image_encode_host(ctx, accum.data(), W, H, p.spp, &io, nullptr, &bytes, nullptr);
            if (st == MC_OK) {
                img.resize((size_t)bytes);
                st = mc_image_encode_host(ctx, accum.data(), W, H, p.spp, &io, img.data(), &bytes, &chosen);
            }
            if (st != MC_OK) {
                rc = fail("mc_image_encode_host", st);
            } else {
                if (o.exposure <= 0.f) std::printf("Auto exposure: %.3f\n", chosen);  // PT:4358
                char head[64];
                size_t headBytes = 0;
                if (io.format == MC_IMAGE_RGB8) headBytes = (size_t)std::snprintf(head, sizeof(head), "P6\n%d %d\n255\n", W, H);
                if (!write_file(o.out, head, headBytes, img.data(), img.size())) {
                    std::fprintf(stderr, "could not write '%s'\n", o.out.c_str());
                    rc = 1;
                } else {
                    std::printf("wrote %s\n", o.out.c_str());
                }
            }
        }
    }
    cleanup();
    return rc;
}
