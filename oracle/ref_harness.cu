// Oracle harness around the UNMODIFIED reference (test infrastructure only).
//
// This translation unit #includes the reference's src/path_tracer.cu as it is
// (its main() renamed by the preprocessor) and exposes a small C API that the
// parity tests, the golden-fixture scripts and bench.py's reference arm call.
// It never ships with the library and the library never calls it.
//
// Two builds come from this file (oracle/Makefile):
//   libmcref.so         - curand XORWOW, exactly as the reference draws;
//   libmcref_philox.so  - the same reference code drawing from the counter-based
//                         Philox stream of ref_philox_shim.cuh.
//
// The reference has no API; everything here drives its internals the way its
// main() does (path_tracer.cu:4038-4411): finalizeScene, std::sort of the
// PrimitiveRefs, BVH::generateHierarchy, the hot/cold split, init_rng_kernel,
// g_environment upload, renderWithWavefront / trace_sample_kernel.
#ifdef MCREF_PHILOX
#include "ref_philox_shim.cuh"
#endif

#define main monocuda_reference_main
#include MCREF_SOURCE
#undef main

#include <unistd.h>
#include <fcntl.h>
#include "../include/mc_abi.h"

// The library's seeded synthetic scenes, from its host-only generator source
// (monocuda-pt_b200/csrc/mc_scene_gen.cpp, linked into this harness by
// oracle/Makefile): the reference renders byte-identical scenes without the
// library being loaded.
namespace mc_gen {
const char* generate(const mc_scene_desc* desc, mc_scene_host* out, mc_status* status);
void free_scene(mc_scene_host* s);
}

static_assert(sizeof(triangle) == sizeof(mc_triangle), "triangle layout");
static_assert(sizeof(triangle_hot) == sizeof(mc_triangle_hot), "triangle_hot layout");
static_assert(sizeof(triangle_cold) == sizeof(mc_triangle_cold), "triangle_cold layout");
static_assert(sizeof(sphere) == sizeof(mc_sphere), "sphere layout");
static_assert(sizeof(Light) == sizeof(mc_light), "Light layout");
static_assert(sizeof(BVH_Node) == sizeof(mc_bvh_node), "BVH_Node layout");
static_assert(sizeof(PackedHit) == sizeof(mc_packed_hit), "PackedHit layout");
static_assert(sizeof(Camera) == sizeof(mc_camera), "Camera layout");
static_assert(sizeof(AABB) == sizeof(mc_aabb), "AABB layout");

namespace {

// stdout of the reference (progress lines, scene stats) goes to /dev/null while
// a harness call runs, so callers that print JSON keep a clean stdout.
struct QuietStdout {
    int saved = -1;
    QuietStdout() {
        fflush(stdout);
        saved = dup(1);
        int devnull = open("/dev/null", O_WRONLY);
        if (devnull >= 0) { dup2(devnull, 1); close(devnull); }
    }
    ~QuietStdout() {
        fflush(stdout);
        if (saved >= 0) { dup2(saved, 1); close(saved); }
    }
};

#define MCREF_TRY(call)                                                        \
    do {                                                                       \
        cudaError_t e__ = (call);                                              \
        if (e__ != cudaSuccess) {                                              \
            std::fprintf(stderr, "mcref: %s failed: %s\n", #call, cudaGetErrorString(e__)); \
            return 2;                                                          \
        }                                                                      \
    } while (0)

struct RefState {
    bool ready = false;
    hostScene scene;
    BVH bvh;
    sphere* d_spheres = nullptr;
    triangle_hot* d_hot = nullptr;
    triangle_cold* d_cold = nullptr;
    Light* d_lights = nullptr;
    int sphereCount = 0, triangleCount = 0, lightCount = 0;
    bool sceneHasMedium = false;
    cudaArray_t envArray = nullptr;
    cudaTextureObject_t envTexture = 0;
    float* d_rowCdf = nullptr;
    float* d_colCdf = nullptr;
};
RefState g_ref;

void copyScene(hostScene& scene, const mc_triangle* tris, int nt, const mc_sphere* sph, int ns) {
    scene = hostScene();
    scene.triangles.resize(nt);
    if (nt) std::memcpy(scene.triangles.data(), tris, sizeof(triangle) * (size_t)nt);
    scene.spheres.resize(ns);
    if (ns) std::memcpy(scene.spheres.data(), sph, sizeof(sphere) * (size_t)ns);
}

// main()'s sort (path_tracer.cu:4223-4226), verbatim in behaviour: std::sort by
// mortonCode with a strict less-than, which is not stable.
void referenceSort(hostScene& scene) {
    std::sort(scene.primitiveRefs.begin(), scene.primitiveRefs.end(),
              [](const PrimitiveRef& a, const PrimitiveRef& b) { return a.mortonCode < b.mortonCode; });
}

void freeDevice() {
    if (g_ref.d_spheres) cudaFree(g_ref.d_spheres);
    if (g_ref.d_hot) cudaFree(g_ref.d_hot);
    if (g_ref.d_cold) cudaFree(g_ref.d_cold);
    if (g_ref.d_lights) cudaFree(g_ref.d_lights);
    if (g_ref.envTexture) cudaDestroyTextureObject(g_ref.envTexture);
    if (g_ref.envArray) cudaFreeArray(g_ref.envArray);
    if (g_ref.d_rowCdf) cudaFree(g_ref.d_rowCdf);
    if (g_ref.d_colCdf) cudaFree(g_ref.d_colCdf);
    if (g_ref.bvh.d_internalNodes || g_ref.bvh.d_leafNode) g_ref.bvh.free();
    g_ref = RefState();
}

__global__ void harnessAnyHitKernel(BVH bvh, const sphere* spheres, TriangleView triangles, const float* rays,
                                    const float* tmax, int n, int* occluded) {
    int i = threadIdx.x + blockIdx.x * blockDim.x;
    if (i >= n) return;
    vec3 o(rays[i], rays[n + i], rays[2 * n + i]);
    vec3 d(rays[3 * n + i], rays[4 * n + i], rays[5 * n + i]);
    float t = rays[6 * n + i];
    occluded[i] = bvh.traverseAnyHit(o, d, t, spheres, triangles, tmax[i]) ? 1 : 0;
}

#ifdef MCREF_PHILOX
// Before each sample: the counter-based stream of (pixel, sample) starts at draw 0.
__global__ void harnessPhiloxSampleKernel(curandState* states, int count, unsigned int sample) {
    int i = threadIdx.x + blockIdx.x * blockDim.x;
    if (i >= count) return;
    states[i].sample = sample;
    states[i].draw = 0;
}
#endif

}  // namespace

extern "C" {

int mcref_is_philox(void) {
#ifdef MCREF_PHILOX
    return 1;
#else
    return 0;
#endif
}

// Camera::initialize (path_tracer.cu:1610-1631) on the host.
int mcref_camera_initialize(mc_camera* cam) {
    Camera c;
    std::memcpy(&c, cam, sizeof(Camera));
    c.initialize();
    std::memcpy(cam, &c, sizeof(Camera));
    return 0;
}

// finalizeScene (path_tracer.cu:1930-1987) and main()'s sort (4223-4233), host only.
// Outputs (all host, n = ns + nt entries unless noted):
//   codes_ref_order - Morton code of each PrimitiveRef before sorting
//   sorted_codes/ids/types/bounds - the SoA split of main() (4228-4233)
//   perm - for each sorted slot, its position in the unsorted PrimitiveRef list
//   tri_bounds - triangle::aabb after calculate_bounding_box (nt entries)
//   lights - the light list (capacity nt), *n_lights its length
int mcref_finalize_and_sort(const mc_triangle* tris, int nt, const mc_sphere* sph, int ns,
                            uint32_t* codes_ref_order, uint32_t* sorted_codes, int32_t* sorted_ids,
                            int32_t* sorted_types, int32_t* perm, mc_aabb* sorted_bounds,
                            mc_aabb* scene_bounds, mc_aabb* tri_bounds, mc_light* lights, int32_t* n_lights) {
    QuietStdout quiet;
    hostScene scene;
    copyScene(scene, tris, nt, sph, ns);
    finalizeScene(scene);
    int n = (int)scene.primitiveRefs.size();
    for (int i = 0; i < n; i++)
        if (codes_ref_order) codes_ref_order[i] = scene.primitiveRefs[i].mortonCode;
    referenceSort(scene);
    for (int i = 0; i < n; i++) {
        const PrimitiveRef& r = scene.primitiveRefs[i];
        if (sorted_codes) sorted_codes[i] = r.mortonCode;
        if (sorted_ids) sorted_ids[i] = r.primitiveIndex;
        if (sorted_types) sorted_types[i] = r.primitiveType;
        if (perm) perm[i] = r.primitiveType == 0 ? r.primitiveIndex : ns + r.primitiveIndex;
        if (sorted_bounds) std::memcpy(&sorted_bounds[i], &r.bounds, sizeof(AABB));
    }
    if (scene_bounds) std::memcpy(scene_bounds, &scene.bounds, sizeof(AABB));
    if (tri_bounds)
        for (int i = 0; i < nt; i++) std::memcpy(&tri_bounds[i], &scene.triangles[i].aabb, sizeof(AABB));
    if (n_lights) *n_lights = (int)scene.lights.size();
    if (lights && !scene.lights.empty()) std::memcpy(lights, scene.lights.data(), sizeof(Light) * scene.lights.size());
    return 0;
}

// BVH::generateHierarchy (path_tracer.cu:1063-1090) on given sorted arrays.
// Host in/out. internal_out: n-1 nodes, leaves_out: n nodes.
int mcref_build_bvh(const uint32_t* sorted_codes, const int32_t* sorted_ids, const int32_t* sorted_types,
                    const mc_aabb* sorted_bounds, int n, mc_bvh_node* internal_out, mc_bvh_node* leaves_out) {
    if (n < 2) return 1;
    // The reference's kernels trust their input (an unsorted code array gives a
    // malformed tree whose refit indexes out of bounds): check it on the host.
    for (int i = 1; i < n; i++)
        if (sorted_codes[i] < sorted_codes[i - 1]) return 4;
    for (int i = 0; i < n; i++)
        if (sorted_ids[i] < 0 || (sorted_types[i] != 0 && sorted_types[i] != 1)) return 4;
    unsigned int* d_codes = nullptr; int* d_ids = nullptr; AABB* d_bounds = nullptr; int* d_types = nullptr;
    MCREF_TRY(cudaMalloc(&d_codes, n * sizeof(unsigned int)));
    MCREF_TRY(cudaMalloc(&d_ids, n * sizeof(int)));
    MCREF_TRY(cudaMalloc(&d_bounds, n * sizeof(AABB)));
    MCREF_TRY(cudaMalloc(&d_types, n * sizeof(int)));
    MCREF_TRY(cudaMemcpy(d_codes, sorted_codes, n * sizeof(unsigned int), cudaMemcpyHostToDevice));
    MCREF_TRY(cudaMemcpy(d_ids, sorted_ids, n * sizeof(int), cudaMemcpyHostToDevice));
    MCREF_TRY(cudaMemcpy(d_bounds, sorted_bounds, n * sizeof(AABB), cudaMemcpyHostToDevice));
    MCREF_TRY(cudaMemcpy(d_types, sorted_types, n * sizeof(int), cudaMemcpyHostToDevice));
    BVH bvh;
    bvh.generateHierarchy(d_codes, d_ids, d_bounds, d_types, n);
    MCREF_TRY(cudaMemcpy(internal_out, bvh.d_internalNodes, (size_t)(n - 1) * sizeof(BVH_Node), cudaMemcpyDeviceToHost));
    MCREF_TRY(cudaMemcpy(leaves_out, bvh.d_leafNode, (size_t)n * sizeof(BVH_Node), cudaMemcpyDeviceToHost));
    bvh.free();
    cudaFree(d_codes); cudaFree(d_ids); cudaFree(d_bounds); cudaFree(d_types);
    return 0;
}

// Uploads a scene the way main() does (path_tracer.cu:4188-4303): environment
// map (PFM path replaced by an RGBA array, top row first), sort, BVH, spheres,
// hot/cold split, lights. env_rgba may be NULL (no environment).
int mcref_scene_upload(const mc_triangle* tris, int nt, const mc_sphere* sph, int ns, const float* env_rgba,
                       int env_w, int env_h, float env_intensity, float env_rotation_degrees) {
    QuietStdout quiet;
    freeDevice();
    copyScene(g_ref.scene, tris, nt, sph, ns);
    finalizeScene(g_ref.scene);

    EnvironmentMap env = {0, 0, env_intensity, env_rotation_degrees * MONOCUDA_PI / 180.0f, nullptr, nullptr, 0, 0, 0.0f};
    if (env_rgba && env_w > 0 && env_h > 0) {
        std::vector<float> pixels(env_rgba, env_rgba + (size_t)env_w * env_h * 4);
        g_ref.envTexture = createEnvironmentTexture(pixels, env_w, env_h, g_ref.envArray);
        env.texture = g_ref.envTexture;
        env.enabled = 1;
        std::vector<float> rowCdf, colCdf;
        buildEnvironmentSamplingTables(pixels, env_w, env_h, rowCdf, colCdf, env.totalWeight);
        MCREF_TRY(cudaMalloc(&g_ref.d_rowCdf, rowCdf.size() * sizeof(float)));
        MCREF_TRY(cudaMalloc(&g_ref.d_colCdf, colCdf.size() * sizeof(float)));
        MCREF_TRY(cudaMemcpy(g_ref.d_rowCdf, rowCdf.data(), rowCdf.size() * sizeof(float), cudaMemcpyHostToDevice));
        MCREF_TRY(cudaMemcpy(g_ref.d_colCdf, colCdf.data(), colCdf.size() * sizeof(float), cudaMemcpyHostToDevice));
        env.rowCdf = g_ref.d_rowCdf;
        env.columnCdf = g_ref.d_colCdf;
        env.width = env_w;
        env.height = env_h;
    }
    MCREF_TRY(cudaMemcpyToSymbol(g_environment, &env, sizeof(EnvironmentMap)));

    referenceSort(g_ref.scene);
    int n = (int)g_ref.scene.primitiveRefs.size();
    if (n < 2) return 1;
    std::vector<unsigned int> codes(n);
    std::vector<int> ids(n), types(n);
    std::vector<AABB> bounds(n);
    for (int i = 0; i < n; i++) {
        codes[i] = g_ref.scene.primitiveRefs[i].mortonCode;
        ids[i] = g_ref.scene.primitiveRefs[i].primitiveIndex;
        bounds[i] = g_ref.scene.primitiveRefs[i].bounds;
        types[i] = g_ref.scene.primitiveRefs[i].primitiveType;
    }
    unsigned int* d_codes; int* d_ids; AABB* d_bounds; int* d_types;
    MCREF_TRY(cudaMalloc(&d_codes, n * sizeof(unsigned int)));
    MCREF_TRY(cudaMalloc(&d_ids, n * sizeof(int)));
    MCREF_TRY(cudaMalloc(&d_bounds, n * sizeof(AABB)));
    MCREF_TRY(cudaMalloc(&d_types, n * sizeof(int)));
    MCREF_TRY(cudaMemcpy(d_codes, codes.data(), n * sizeof(unsigned int), cudaMemcpyHostToDevice));
    MCREF_TRY(cudaMemcpy(d_ids, ids.data(), n * sizeof(int), cudaMemcpyHostToDevice));
    MCREF_TRY(cudaMemcpy(d_bounds, bounds.data(), n * sizeof(AABB), cudaMemcpyHostToDevice));
    MCREF_TRY(cudaMemcpy(d_types, types.data(), n * sizeof(int), cudaMemcpyHostToDevice));
    g_ref.bvh.generateHierarchy(d_codes, d_ids, d_bounds, d_types, n);
    cudaFree(d_codes); cudaFree(d_ids); cudaFree(d_bounds); cudaFree(d_types);

    g_ref.sphereCount = ns;
    MCREF_TRY(cudaMalloc(&g_ref.d_spheres, (size_t)(ns > 0 ? ns : 1) * sizeof(sphere)));
    if (ns) MCREF_TRY(cudaMemcpy(g_ref.d_spheres, g_ref.scene.spheres.data(), ns * sizeof(sphere), cudaMemcpyHostToDevice));
    g_ref.triangleCount = nt;
    std::vector<triangle_hot> hot(nt);
    std::vector<triangle_cold> cold(nt);
    for (int i = 0; i < nt; i++) {
        const triangle& t = g_ref.scene.triangles[i];
        hot[i] = triangle_hot(t.v0, t.v1, t.v2);
        cold[i] = triangle_cold(t.uv0, t.uv1, t.uv2, t.n0, t.n1, t.n2, t.mat, t.aabb);
    }
    MCREF_TRY(cudaMalloc(&g_ref.d_hot, (size_t)(nt > 0 ? nt : 1) * sizeof(triangle_hot)));
    MCREF_TRY(cudaMalloc(&g_ref.d_cold, (size_t)(nt > 0 ? nt : 1) * sizeof(triangle_cold)));
    if (nt) {
        MCREF_TRY(cudaMemcpy(g_ref.d_hot, hot.data(), nt * sizeof(triangle_hot), cudaMemcpyHostToDevice));
        MCREF_TRY(cudaMemcpy(g_ref.d_cold, cold.data(), nt * sizeof(triangle_cold), cudaMemcpyHostToDevice));
    }
    g_ref.lightCount = (int)g_ref.scene.lights.size();
    MCREF_TRY(cudaMalloc(&g_ref.d_lights, (size_t)(g_ref.lightCount > 0 ? g_ref.lightCount : 1) * sizeof(Light)));
    if (g_ref.lightCount)
        MCREF_TRY(cudaMemcpy(g_ref.d_lights, g_ref.scene.lights.data(), g_ref.lightCount * sizeof(Light), cudaMemcpyHostToDevice));
    bool medium = false;
    for (const sphere& s : g_ref.scene.spheres) if (s.mat.type == MaterialType::Isotropic) medium = true;
    for (const triangle& t : g_ref.scene.triangles) if (t.mat.type == MaterialType::Isotropic) medium = true;
    g_ref.sceneHasMedium = medium;
    g_ref.ready = true;
    return 0;
}

int mcref_scene_release(void) {
    freeDevice();
    return 0;
}

// Ray set through the reference's own kernels. rays: host SoA (7*n floats:
// ox, oy, oz, dx, dy, dz, time). mode 0 = extendKernelPersistent
// (path_tracer.cu:3416), 1 = extendKernel (3376), 2 = any hit (traverseAnyHit,
// 1152) with tmax. Outputs are host arrays of n entries.
int mcref_trace(const float* rays, int n, int mode, const float* tmax, mc_packed_hit* hits, int32_t* occluded) {
    if (!g_ref.ready || n <= 0) return 1;
    TriangleView tv{g_ref.d_hot, g_ref.d_cold};
    if (mode == 2) {
        float* d_rays; float* d_tmax; int* d_occ;
        MCREF_TRY(cudaMalloc(&d_rays, (size_t)7 * n * sizeof(float)));
        MCREF_TRY(cudaMalloc(&d_tmax, (size_t)n * sizeof(float)));
        MCREF_TRY(cudaMalloc(&d_occ, (size_t)n * sizeof(int)));
        MCREF_TRY(cudaMemcpy(d_rays, rays, (size_t)7 * n * sizeof(float), cudaMemcpyHostToDevice));
        MCREF_TRY(cudaMemcpy(d_tmax, tmax, (size_t)n * sizeof(float), cudaMemcpyHostToDevice));
        harnessAnyHitKernel<<<(n + 255) / 256, 256>>>(g_ref.bvh, g_ref.d_spheres, tv, d_rays, d_tmax, n, d_occ);
        MCREF_TRY(cudaGetLastError());
        MCREF_TRY(cudaMemcpy(occluded, d_occ, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost));
        cudaFree(d_rays); cudaFree(d_tmax); cudaFree(d_occ);
        return 0;
    }
    PathStateBuffers ps;
    HitResultBuffers hr;
    PathQueue q;
    allocatePathStateBuffers(ps, n);
    allocateHitResultBuffers(hr, n);
    allocatePathQueue(q, n);
    MCREF_TRY(cudaMemcpy(ps.rayOriginX, rays + 0 * (size_t)n, n * sizeof(float), cudaMemcpyHostToDevice));
    MCREF_TRY(cudaMemcpy(ps.rayOriginY, rays + 1 * (size_t)n, n * sizeof(float), cudaMemcpyHostToDevice));
    MCREF_TRY(cudaMemcpy(ps.rayOriginZ, rays + 2 * (size_t)n, n * sizeof(float), cudaMemcpyHostToDevice));
    MCREF_TRY(cudaMemcpy(ps.rayDirectionX, rays + 3 * (size_t)n, n * sizeof(float), cudaMemcpyHostToDevice));
    MCREF_TRY(cudaMemcpy(ps.rayDirectionY, rays + 4 * (size_t)n, n * sizeof(float), cudaMemcpyHostToDevice));
    MCREF_TRY(cudaMemcpy(ps.rayDirectionZ, rays + 5 * (size_t)n, n * sizeof(float), cudaMemcpyHostToDevice));
    MCREF_TRY(cudaMemcpy(ps.rayTime, rays + 6 * (size_t)n, n * sizeof(float), cudaMemcpyHostToDevice));
    std::vector<int> identity(n);
    for (int i = 0; i < n; i++) identity[i] = i;
    MCREF_TRY(cudaMemcpy(q.pathIndices, identity.data(), n * sizeof(int), cudaMemcpyHostToDevice));
    MCREF_TRY(cudaMemcpy(q.itemCount, &n, sizeof(int), cudaMemcpyHostToDevice));
    int blockCount = (n + 255) / 256;
    if (mode == 0) {
        int* counter; MCREF_TRY(cudaMalloc(&counter, sizeof(int)));
        MCREF_TRY(cudaMemset(counter, 0, sizeof(int)));
        int dev = 0, sms = 0, per = 0;
        MCREF_TRY(cudaGetDevice(&dev));
        MCREF_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        MCREF_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, extendKernelPersistent, 256, 0));
        int blocks = std::min(blockCount, sms * per);
        extendKernelPersistent<<<blocks, 256>>>(g_ref.bvh, g_ref.d_spheres, tv, ps, hr, q, counter);
        MCREF_TRY(cudaGetLastError());
        MCREF_TRY(cudaDeviceSynchronize());
        cudaFree(counter);
    } else {
        extendKernel<<<blockCount, 256>>>(g_ref.bvh, g_ref.d_spheres, tv, ps, hr, q);
        MCREF_TRY(cudaGetLastError());
        MCREF_TRY(cudaDeviceSynchronize());
    }
    MCREF_TRY(cudaMemcpy(hits, hr.packedHits, (size_t)n * sizeof(PackedHit), cudaMemcpyDeviceToHost));
    freePathQueue(q);
    freeHitResultBuffers(hr);
    freePathStateBuffers(ps);
    return 0;
}

// Renders with the reference's kernels.
//   mode 0: megakernel (trace_sample_kernel + resolve_kernel per sample, 4331-4351)
//   mode 1: wavefront, mode 2: wavefront + persistent extend
//   unmodified = 1 (XORWOW build only): call renderWithWavefront itself (3757)
//   unmodified = 0: the harness's copy of renderWithWavefront's launch sequence,
//     which also reads each bounce's shadow-queue size (ray counting) and, in
//     the Philox build, restarts the counter-based stream per (pixel, sample).
// cam: fields as main() sets them; Camera::initialize is applied here.
// accum_out: host W*H*3 floats (the accumulation buffer after all samples).
// stats_out (may be NULL): [0] extend rays, [1] shadow rays, [2] render ms.
int mcref_render(const mc_camera* cam_in, int W, int H, int spp, int max_depth, int mode, unsigned long long seed,
                 int first_sample, int unmodified, float* accum_out, double* stats_out) {
    if (!g_ref.ready || W <= 0 || H <= 0 || spp <= 0) return 1;
    QuietStdout quiet;
    Camera cam;
    std::memcpy(&cam, cam_in, sizeof(Camera));
    cam.aspect_ratio = W / float(H);
    cam.image_width = W;
    cam.max_depth = max_depth;
    cam.samples_per_pixel = spp;
    cam.initialize();

    int pixels = W * H;
    int dev = 0;
    cudaDeviceProp props;
    MCREF_TRY(cudaGetDevice(&dev));
    MCREF_TRY(cudaGetDeviceProperties(&props, dev));
    bool wave = mode != 0;
    dim3 block = wave ? chooseImageBlockShape(generateCameraRaysKernel, props) : chooseImageBlockShape(trace_sample_kernel, props);
    dim3 grid = chooseImageGridShape(block, W, H, props);

    vec3* d_accum; vec3* d_frame; curandState* d_rng;
    MCREF_TRY(cudaMalloc(&d_accum, pixels * sizeof(vec3)));
    MCREF_TRY(cudaMalloc(&d_frame, pixels * sizeof(vec3)));
    MCREF_TRY(cudaMalloc(&d_rng, pixels * sizeof(curandState)));
    MCREF_TRY(cudaMemset(d_accum, 0, pixels * sizeof(vec3)));
    MCREF_TRY(cudaMemset(d_frame, 0, pixels * sizeof(vec3)));
    init_rng_kernel<<<grid, block>>>(d_rng, W, H, seed);
    MCREF_TRY(cudaGetLastError());
    MCREF_TRY(cudaDeviceSynchronize());

    TriangleView tv{g_ref.d_hot, g_ref.d_cold};
    double extendRays = 0, shadowRays = 0;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto t0 = std::chrono::steady_clock::now();
    cudaEventRecord(e0);

    if (!wave) {
        for (int s = 0; s < spp; s++) {
#ifdef MCREF_PHILOX
            harnessPhiloxSampleKernel<<<(pixels + 255) / 256, 256>>>(d_rng, pixels, (unsigned)(first_sample + s));
#endif
            trace_sample_kernel<<<grid, block>>>(d_accum, cam, g_ref.bvh, g_ref.d_spheres, g_ref.sphereCount, tv,
                                                 g_ref.triangleCount, W, H, d_rng, s, g_ref.d_lights, g_ref.lightCount);
            MCREF_TRY(cudaGetLastError());
            MCREF_TRY(cudaDeviceSynchronize());
            resolve_kernel<<<grid, block>>>(d_accum, d_frame, W, H, s + 1, ToneMapOption::None, 1.0f);
            MCREF_TRY(cudaGetLastError());
            MCREF_TRY(cudaDeviceSynchronize());
        }
    } else {
        WavefrontRenderContext ctx;
        ctx.camera = cam;
        ctx.bvh = g_ref.bvh;
        ctx.spheres = g_ref.d_spheres;
        ctx.sphereCount = g_ref.sphereCount;
        ctx.triangles = tv;
        ctx.triangleCount = g_ref.triangleCount;
        ctx.lights = g_ref.d_lights;
        ctx.lightCount = g_ref.lightCount;
        ctx.accumBuffer = d_accum;
        ctx.frameBuffer = d_frame;
        ctx.randomNumberStates = d_rng;
        ctx.imageWidth = W;
        ctx.imageHeight = H;
        ctx.gridDimensions = grid;
        ctx.blockDimensions = block;
        ctx.toneMap = ToneMapOption::None;
        ctx.exposure = 1.f;
        ctx.usePersistentThreads = (mode == 2);
        ctx.sceneHasMedium = g_ref.sceneHasMedium;
#ifndef MCREF_PHILOX
        if (unmodified) {
            renderWithWavefront(ctx);
        } else
#endif
        {
            // Same allocations and launch order as renderWithWavefront (3757-3840).
            int pathCapacity = pixels;
            PathStateBuffers pathState; HitResultBuffers hitResults; PathQueue currentQueue, nextQueue; ShadowRayQueue shadowQueue;
            allocatePathStateBuffers(pathState, pathCapacity);
            allocateHitResultBuffers(hitResults, pathCapacity);
            allocatePathQueue(currentQueue, pathCapacity);
            allocatePathQueue(nextQueue, pathCapacity);
            allocateShadowRayQueue(shadowQueue, pathCapacity);
            int* workCounter = nullptr;
            int persistentBlocks = 0;
            if (ctx.usePersistentThreads) {
                MCREF_TRY(cudaMalloc(&workCounter, sizeof(int)));
                int sms = 0, per = 0;
                MCREF_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
                MCREF_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, extendKernelPersistent, 256, 0));
                persistentBlocks = sms * per;
            }
            for (int s = 0; s < spp; ++s) {
#ifdef MCREF_PHILOX
                harnessPhiloxSampleKernel<<<(pixels + 255) / 256, 256>>>(d_rng, pixels, (unsigned)(first_sample + s));
#endif
                generateCameraRaysKernel<<<grid, block>>>(cam, W, H, d_rng, pathState, currentQueue);
                MCREF_TRY(cudaGetLastError());
                MCREF_TRY(cudaDeviceSynchronize());
                int active = pathCapacity;
                MCREF_TRY(cudaMemcpy(currentQueue.itemCount, &active, sizeof(int), cudaMemcpyHostToDevice));
                for (int depth = 0; depth < max_depth; ++depth) {
                    if (active == 0) break;
                    extendRays += active;
                    MCREF_TRY(cudaMemset(nextQueue.itemCount, 0, sizeof(int)));
                    MCREF_TRY(cudaMemset(shadowQueue.itemCount, 0, sizeof(int)));
                    int blockSize = 256;
                    int blockCount = (active + blockSize - 1) / blockSize;
                    if (ctx.usePersistentThreads) {
                        MCREF_TRY(cudaMemset(workCounter, 0, sizeof(int)));
                        extendKernelPersistent<<<std::min(blockCount, persistentBlocks), blockSize>>>(
                            g_ref.bvh, g_ref.d_spheres, tv, pathState, hitResults, currentQueue, workCounter);
                    } else {
                        extendKernel<<<blockCount, blockSize>>>(g_ref.bvh, g_ref.d_spheres, tv, pathState, hitResults, currentQueue);
                    }
                    MCREF_TRY(cudaGetLastError());
                    MCREF_TRY(cudaDeviceSynchronize());
                    shadeKernel<<<blockCount, blockSize>>>(depth, cam.backround_color, cam.russianRouletteCap, g_ref.d_spheres, tv,
                                                           g_ref.d_lights, g_ref.lightCount, d_rng, pathState, hitResults,
                                                           currentQueue, nextQueue, shadowQueue);
                    MCREF_TRY(cudaGetLastError());
                    MCREF_TRY(cudaDeviceSynchronize());
                    shadowKernel<<<blockCount, blockSize>>>(g_ref.bvh, g_ref.d_spheres, tv, pathState, shadowQueue,
                                                            ctx.sceneHasMedium, d_rng);
                    MCREF_TRY(cudaGetLastError());
                    MCREF_TRY(cudaDeviceSynchronize());
                    int shadowCount = 0;
                    MCREF_TRY(cudaMemcpy(&shadowCount, shadowQueue.itemCount, sizeof(int), cudaMemcpyDeviceToHost));
                    shadowRays += shadowCount;
                    MCREF_TRY(cudaMemcpy(&active, nextQueue.itemCount, sizeof(int), cudaMemcpyDeviceToHost));
                    std::swap(currentQueue, nextQueue);
                }
                finalizeSampleKernel<<<grid, block>>>(d_accum, W, H, pathState);
                MCREF_TRY(cudaGetLastError());
                MCREF_TRY(cudaDeviceSynchronize());
                resolve_kernel<<<grid, block>>>(d_accum, d_frame, W, H, s + 1, ToneMapOption::None, 1.0f);
                MCREF_TRY(cudaGetLastError());
                MCREF_TRY(cudaDeviceSynchronize());
            }
            freeShadowRayQueue(shadowQueue);
            if (workCounter) cudaFree(workCounter);
            freePathQueue(nextQueue);
            freePathQueue(currentQueue);
            freeHitResultBuffers(hitResults);
            freePathStateBuffers(pathState);
        }
    }
    cudaEventRecord(e1);
    MCREF_TRY(cudaEventSynchronize(e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    double hostMs = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    (void)hostMs;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (accum_out) MCREF_TRY(cudaMemcpy(accum_out, d_accum, pixels * sizeof(vec3), cudaMemcpyDeviceToHost));
    if (stats_out) { stats_out[0] = extendRays; stats_out[1] = shadowRays; stats_out[2] = ms; }
    cudaFree(d_accum); cudaFree(d_frame); cudaFree(d_rng);
    return 0;
}

// resolve_kernel (path_tracer.cu:3092-3100) on a host accumulation buffer,
// with the exposure of computeAutoExposure (3121-3132) when auto_exposure is
// set, launched with main()'s wavefront block and grid shapes (4101-4103),
// then the 8-bit encoding main() applies before writing the PNG (4363-4380,
// restated here: it is inline in main()). Outputs (host, may be NULL):
// frame W*H*3 floats, rgb8 W*H*3 bytes, *chosen the exposure used.
int mcref_resolve(const float* accum_in, int W, int H, int samples, int tonemap, float exposure, int auto_exposure,
                  float* frame_out, unsigned char* rgb8_out, float* chosen) {
    if (W <= 0 || H <= 0 || samples <= 0 || tonemap < 0 || tonemap > 2) return 1;
    QuietStdout quiet;
    int dev = 0;
    cudaDeviceProp props;
    MCREF_TRY(cudaGetDevice(&dev));
    MCREF_TRY(cudaGetDeviceProperties(&props, dev));
    dim3 block = chooseImageBlockShape(generateCameraRaysKernel, props);
    dim3 grid = chooseImageGridShape(block, W, H, props);
    const size_t pixels = (size_t)W * H;
    vec3* d_accum; vec3* d_frame;
    MCREF_TRY(cudaMalloc(&d_accum, pixels * sizeof(vec3)));
    MCREF_TRY(cudaMalloc(&d_frame, pixels * sizeof(vec3)));
    MCREF_TRY(cudaMemcpy(d_accum, accum_in, pixels * sizeof(vec3), cudaMemcpyHostToDevice));
    float e = exposure;
    if (auto_exposure) e = computeAutoExposure(d_accum, W, H, samples, grid, block);
    resolve_kernel<<<grid, block>>>(d_accum, d_frame, W, H, samples, (ToneMapOption)tonemap, e);
    MCREF_TRY(cudaGetLastError());
    std::vector<vec3> frame(pixels);
    MCREF_TRY(cudaMemcpy(frame.data(), d_frame, pixels * sizeof(vec3), cudaMemcpyDeviceToHost));
    cudaFree(d_accum);
    cudaFree(d_frame);
    if (frame_out) std::memcpy(frame_out, frame.data(), pixels * sizeof(vec3));
    if (rgb8_out) {
        for (size_t p = 0; p < pixels; p++) {
            const float c[3] = {frame[p].x, frame[p].y, frame[p].z};
            for (int k = 0; k < 3; k++) {
                float f = std::isfinite(c[k]) ? fminf(fmaxf(c[k], 0.0f), 1.0f) : 0.0f;
                rgb8_out[3 * p + k] = (unsigned char)(255.99f * f);
            }
        }
    }
    if (chosen) *chosen = e;
    return 0;
}

// loadObject (path_tracer.cu:2644-2859) into an empty scene; copies up to
// `capacity` triangles out, *count = the number loaded. Returns 0 when the
// reference reports success, 3 when it returns false.
int mcref_load_object(const char* path, const mc_material* mat, float tx, float ty, float tz, float scale, float rot,
                      mc_triangle* out, int capacity, int* count) {
    QuietStdout quiet;
    hostScene scene;
    Material m;
    static_assert(sizeof(Material) == sizeof(mc_material), "Material layout");
    std::memcpy(&m, mat, sizeof(Material));
    bool ok = loadObject(scene, path, m, vec3(tx, ty, tz), scale, rot);
    const int n = (int)scene.triangles.size();
    if (count) *count = n;
    for (int i = 0; i < n && i < capacity; i++) std::memcpy(&out[i], &scene.triangles[i], sizeof(triangle));
    return ok ? 0 : 3;
}

// setup_scene(SceneChoice::Cloud) (path_tracer.cu:2486-2524, buildCloudScene
// 1849-1891) for a grid with these world bounds and maximum, as main() leaves
// the globals after loading one (4066-4076): grid_pointer is only stored in
// the medium's material. sun != 0: no --env (the sun quad is built). Copies
// up to the capacities out; returns 0, or 3 when the scene is empty.
int mcref_cloud_scene(const float* world_min, const float* world_max, float maximum, unsigned long long grid_pointer,
                      int sun, mc_triangle* tris, int tri_capacity, int* tri_count, mc_sphere* spheres,
                      int sphere_capacity, int* sphere_count) {
    QuietStdout quiet;
    for (int a = 0; a < 3; a++) {
        g_volumeGrid.worldMinimum[a] = world_min[a];
        g_volumeGrid.worldMaximum[a] = world_max[a];
    }
    g_volumeGrid.maximumDensity = maximum;
    g_volumeDeviceGrid = reinterpret_cast<const nanovdb::FloatGrid*>(grid_pointer);
    g_environmentEnabled = sun == 0;
    g_phaseGWasSet = false;
    hostScene scene = setup_scene(SceneChoice::Cloud);
    g_volumeDeviceGrid = nullptr;
    g_environmentEnabled = false;
    const int nt = (int)scene.triangles.size(), ns = (int)scene.spheres.size();
    if (tri_count) *tri_count = nt;
    if (sphere_count) *sphere_count = ns;
    for (int i = 0; i < nt && i < tri_capacity; i++) std::memcpy(&tris[i], &scene.triangles[i], sizeof(triangle));
    for (int i = 0; i < ns && i < sphere_capacity; i++) std::memcpy(&spheres[i], &scene.spheres[i], sizeof(sphere));
    return nt + ns > 0 ? 0 : 3;
}

// The grid reading of sampleVolumeDensity (path_tracer.cu:784-789: world to
// index, accessor, order-1 sampler) through the nanovdb stand-in, on the host:
// grid_bytes is a host copy of a grid (64-byte header, then the voxels).
int mcref_grid_sample(const void* grid_bytes, const float* points, int n, float* out) {
    const nanovdb::FloatGrid* grid = reinterpret_cast<const nanovdb::FloatGrid*>(grid_bytes);
    for (int i = 0; i < n; i++) {
        const nanovdb::Vec3f index = grid->worldToIndexF(nanovdb::Vec3f(points[3 * i], points[3 * i + 1], points[3 * i + 2]));
        auto accessor = grid->tree().getAccessor();
        out[i] = nanovdb::math::createSampler<1>(accessor)(index);
    }
    return 0;
}

// loadPfmAsRgba32f (path_tracer.cu:335-368): 0 and the size (and, when rgba is
// not NULL, the RGBA pixels) when the reference accepts the file, 3 when not.
int mcref_load_pfm(const char* path, int* width, int* height, float* rgba) {
    int w = 0, h = 0;
    std::vector<float> pixels;
    if (!loadPfmAsRgba32f(path, w, h, pixels)) return 3;
    if (width) *width = w;
    if (height) *height = h;
    if (rgba) std::memcpy(rgba, pixels.data(), pixels.size() * sizeof(float));
    return 0;
}

// One of the library's seeded synthetic scenes (mc_scene_generate's kinds and
// arguments), host arrays released by mcref_free_scene. Returns 0 or the
// library's status code.
int mcref_generate_scene(int kind, int variant, unsigned long long seed, int triangle_target, mc_scene_host* out) {
    mc_scene_desc d;
    std::memset(&d, 0, sizeof(d));
    d.kind = kind;
    d.variant = variant;
    d.seed = seed;
    d.triangle_target = triangle_target;
    mc_status st = MC_OK;
    if (mc_gen::generate(&d, out, &st)) {
        mc_gen::free_scene(out);
        return (int)st;
    }
    return 0;
}

int mcref_free_scene(mc_scene_host* s) {
    mc_gen::free_scene(s);
    return 0;
}

}  // extern "C"
