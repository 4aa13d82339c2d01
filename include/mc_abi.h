/*
 * mc_abi.h - C ABI of the B200-native MonoCUDA-PT render hot path.
 *
 * Plain C, plain pointers and sizes. Every pointer documented as "device" is a
 * CUDA device pointer on the context's device; "host" pointers are ordinary
 * host memory. No call exits the process: every entry point returns an
 * mc_status, and mc_last_error() gives the message of the last failure on the
 * calling thread.
 *
 * The structs below reproduce the byte layouts of the reference's scene surface
 * (src/path_tracer.cu, "PT" below) so that arrays built for the reference can be
 * handed to this library unchanged. Their sizes and field offsets are pinned by
 * static_asserts at the end of this header (C11 or C++11).
 */
#ifndef MC_ABI_H
#define MC_ABI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
#define MC_ALIGNAS(n) alignas(n)
extern "C" {
#else
#define MC_ALIGNAS(n) _Alignas(n)
#endif

#if defined(_WIN32)
#define MC_API __declspec(dllexport)
#else
#define MC_API __attribute__((visibility("default")))
#endif

/* ------------------------------------------------------------------------- */
/* Status codes. The reference calls exit() on any CUDA error (PT:55-69).     */
/* ------------------------------------------------------------------------- */
typedef enum mc_status {
    MC_OK = 0,
    MC_ERR_INVALID = 1,         /* bad argument (null pointer, size out of range, ...) */
    MC_ERR_CUDA = 2,            /* a CUDA runtime call failed */
    MC_ERR_OOM = 3,             /* device allocation failed */
    MC_ERR_STACK_OVERFLOW = 4,  /* a traversal stack would have overflowed; the ray was abandoned */
    MC_ERR_QUEUE_OVERFLOW = 5,  /* a queue append went past its capacity; the entry was dropped */
    MC_ERR_TIMEOUT = 6,         /* a bounded device wait ran out */
    MC_ERR_BUDGET = 7,          /* a request does not fit the server's HBM budget */
    MC_ERR_CANCELLED = 8,       /* a server request was cancelled */
    MC_ERR_NOT_FOUND = 9,       /* unknown handle / id */
    MC_ERR_UNSUPPORTED = 10     /* feature compiled out or not available (e.g. no GPU) */
} mc_status;

/* ------------------------------------------------------------------------- */
/* Scene surface (reference layouts).                                          */
/* ------------------------------------------------------------------------- */
typedef struct mc_vec3 { float x, y, z; } mc_vec3;          /* PT:105 vec3 */
typedef struct mc_vec2 { float x, y; } mc_vec2;             /* PT:161 vec2 */

/* PT:612-625 AABB: 32 bytes, 16-byte aligned (two 16-byte vector loads). */
typedef struct mc_aabb {
    MC_ALIGNAS(16) mc_vec3 lo;
    float pad0;
    mc_vec3 hi;
    float pad1;
} mc_aabb;

/* PT:191-199 Texture */
enum { MC_TEX_SOLID = 0, MC_TEX_CHECKER = 1, MC_TEX_IMAGE = 2 };
typedef struct mc_texture {
    int32_t type;
    mc_vec3 color_a;
    mc_vec3 color_b;
    float scale;
    uint64_t image;             /* cudaTextureObject_t for MC_TEX_IMAGE */
} mc_texture;

/* PT:482-496 Material */
enum {
    MC_MAT_LAMBERTIAN = 0,
    MC_MAT_DIELECTRIC = 1,
    MC_MAT_CONDUCTOR = 2,
    MC_MAT_EMISSIVE = 3,
    MC_MAT_ISOTROPIC = 4
};
typedef struct mc_material {
    int32_t type;
    mc_texture albedo;
    mc_vec3 emitted;
    float fuzz;
    float refraction_index;
    float density;
    float phase_g;
    const void* density_grid;   /* device mc_volume_grid (a NanoVDB FloatGrid in the reference) or NULL */
    float grid_max_density;
} mc_material;

/* PT:636-658 triangle (the full host record) */
typedef struct mc_triangle {
    mc_vec3 v0, v1, v2;
    mc_vec2 uv0, uv1, uv2;
    mc_vec3 n0, n1, n2;
    mc_material mat;
    mc_aabb aabb;
} mc_triangle;

/* PT:660-670 triangle_hot: the 36-byte stream the intersector reads */
typedef struct mc_triangle_hot { mc_vec3 v0, v1, v2; } mc_triangle_hot;

/* PT:672-680 triangle_cold */
typedef struct mc_triangle_cold {
    mc_vec2 uv0, uv1, uv2;
    mc_vec3 n0, n1, n2;
    mc_material mat;
    mc_aabb aabb;
} mc_triangle_cold;

/* PT:845-875 sphere */
typedef struct mc_sphere {
    mc_vec3 center;
    mc_vec3 center1;
    uint8_t is_moving;
    float radius;
    mc_material mat;
    mc_aabb aabb;
} mc_sphere;

/* PT:942-947 Light (one emissive triangle) */
typedef struct mc_light {
    mc_triangle_hot tri;
    mc_vec3 emitted;
    float area;
    mc_vec3 normal;
} mc_light;

/* PT:1010-1019 BVH_Node: the reference's binary node layout, used for export
 * and parity checks. The library traverses its own compressed layouts. */
typedef struct mc_bvh_node {
    mc_aabb bounds;
    int32_t left;
    int32_t right;
    uint8_t left_is_leaf;
    uint8_t right_is_leaf;
    int32_t parent;
    int32_t prim;
    uint8_t is_leaf;
} mc_bvh_node;

/* PT:991-996 PackedHit */
typedef struct mc_packed_hit {
    MC_ALIGNAS(16) float t;
    int32_t type;               /* 0 sphere, 1 triangle, -1 none */
    int32_t index;
    int32_t did_hit;
} mc_packed_hit;

/* PT:1581-1631 Camera (fields only). mc_camera_initialize() fills the derived
 * fields exactly like Camera::initialize(). */
typedef struct mc_camera {
    float aspect_ratio;
    int32_t image_width;
    int32_t image_height;
    int32_t samples_per_pixel;
    int32_t max_depth;
    float vfov;
    mc_vec3 look_from;
    mc_vec3 look_at;
    mc_vec3 up;
    mc_vec3 center;
    mc_vec3 pixel00;
    mc_vec3 pixel_delta_u;
    mc_vec3 pixel_delta_v;
    mc_vec3 u, v, w;
    mc_vec3 background;
    float aperture;
    float lens_radius;
    float focus_distance;
    float rr_cap;
} mc_camera;

/* PT:322-333 EnvironmentMap (g_environment). Pointers are device pointers.
 * Maps made by mc_env_create also carry an alias table of the same texel
 * distribution (MC_ENV_SAMPLE_ALIAS), kept by the library beside col_cdf. */
typedef struct mc_env_map {
    uint64_t texture;           /* cudaTextureObject_t (float4, linear, wrap/clamp) */
    int32_t enabled;
    float intensity;
    float rotation;             /* radians */
    const float* row_cdf;       /* height + 1 */
    const float* col_cdf;       /* height * (width + 1) */
    int32_t width;
    int32_t height;
    float total_weight;
} mc_env_map;

/* ------------------------------------------------------------------------- */
/* Library-side handles and parameter blocks.                                  */
/* ------------------------------------------------------------------------- */
typedef struct mc_context mc_context;
typedef struct mc_bvh mc_bvh;

/* Scene as the render path sees it after the reference's upload sequence
 * (PT:4262-4303): every array is a device pointer and stays owned by the caller. */
typedef struct mc_scene_view {
    const mc_sphere* spheres;
    int32_t sphere_count;
    const mc_triangle_hot* tri_hot;
    const mc_triangle_cold* tri_cold;
    int32_t triangle_count;
    const mc_light* lights;
    int32_t light_count;
    int32_t has_medium;         /* PT:4328-4331 sceneHasMedium: MC_MEDIUM_ANY, | MC_MEDIUM_GRID with density grids */
    mc_env_map env;
} mc_scene_view;

enum {
    MC_BVH_LAYOUT_BINARY = 0,   /* children's boxes stored in the parent, 64 B per node */
    MC_BVH_LAYOUT_WIDE4 = 1,    /* 4-wide collapse of the binary tree, exact boxes, 128 B per node */
    MC_BVH_LAYOUT_WIDE4Q = 2    /* the same tree with child boxes quantised to 8 bits per plane
                                   against a per-node frame, rounded outward, 64 B per node */
};

/* The binary tree a wide layout collapses. Every layout keeps the reference's
 * LBVH (Morton codes, Karras hierarchy) for export and parity; hits are the
 * same with either tree (leaves keep the reference's rank for ties). */
enum {
    MC_BVH_BUILDER_CLUSTERED = 0,  /* default: agglomerative clustering of the Morton-sorted leaves by merged
                                      surface area (PLOC), about 40 % fewer node visits per ray */
    MC_BVH_BUILDER_LBVH = 1        /* the reference's LBVH */
};

typedef struct mc_bvh_build_opts {
    /* Optional device array of n = sphere_count + triangle_count ints: the
     * primitive-reference order to use instead of the library's stable radix
     * order (entry k = position in the sphere-then-triangle reference list of
     * the k-th sorted primitive). Lets a caller reproduce the reference's
     * std::sort tie order inside runs of equal Morton codes. NULL = own order. */
    const int32_t* permutation;
    int32_t layout;             /* MC_BVH_LAYOUT_* */
    int32_t keep_reference_nodes; /* keep PT-layout nodes for mc_bvh_export */
    int32_t builder;            /* MC_BVH_BUILDER_*: the binary tree the wide layouts collapse */
    int32_t phase_launches;     /* 1: the clustering rounds and the 4-wide collapse's levels run as one
                                   launch per phase with host checks between them; 0: each loop runs as one
                                   cooperative (persistent) launch where the device supports it. The same
                                   tree either way */
} mc_bvh_build_opts;

typedef struct mc_bvh_info {
    int32_t primitive_count;
    int32_t internal_count;
    int32_t depth;              /* max leaf depth (root = 0) */
    int32_t layout;
    int64_t node_bytes;         /* bytes of the traversal node array */
    int64_t prim_bytes;         /* bytes of the leaf-ordered triangle stream */
    mc_aabb scene_bounds;
    int32_t wide_levels;        /* levels of the 4-wide tree; a ray's traversal stack holds at most
                                   3 entries per level (0: binary layout or not known) */
} mc_bvh_info;

enum {
    MC_RNG_PHILOX = 0,          /* counter-based Philox-4x32-10 keyed by (seed, pixel), counter (sample, draw) */
    MC_RNG_XORWOW = 1           /* curand XORWOW per pixel, curand_init(seed, pixel, 0), state kept across samples */
};

enum {
    MC_ISECT_REFERENCE = 0,     /* the reference's plane + edge test (PT:715-741) */
    MC_ISECT_WATERTIGHT = 1     /* watertight test (Woop, Benthin, Wald 2013) */
};
/* OR into the intersector argument of mc_trace_closest / mc_trace_any: one
 * thread per ray without refill (the reference's plain extendKernel) instead
 * of the persistent refill loop. Results are identical; only scheduling differs. */
#define MC_TRACE_PLAIN 0x100

typedef struct mc_render_params {
    mc_camera camera;           /* initialized; image_width/height set */
    int32_t width;
    int32_t height;
    int32_t spp;                /* samples rendered by this call */
    int32_t first_sample;       /* sample index of the first one (progressive rendering) */
    int32_t max_depth;          /* bounces, 0..MC_MAX_DEPTH (the cloud scene uses 1000, PT:4166) */
    int32_t persistent;         /* PT --persistent: persistent extend kernel */
    int32_t rng;                /* MC_RNG_* */
    uint64_t seed;              /* PT:4297 uses 1234 */
    int32_t intersector;        /* MC_ISECT_* */
    int32_t disable_clamp;      /* 1 = no firefly clamp (guiding MSE studies) */
    int32_t queue_capacity;     /* entries each extend / shadow queue holds; 0 = the wave's paths (every path
                                   fits). Smaller values are a memory or fault-handling test: a bounce whose
                                   queue would overflow keeps the first entries, drops the rest and the call
                                   returns MC_ERR_QUEUE_OVERFLOW (the image is then incomplete) */
    int32_t refill_threshold;   /* idle lanes before a warp refills (PT:3400 uses 8); 0 = 8 */
    int32_t use_graph;          /* capture each sample's bounce sequence in a CUDA graph */
    int32_t instrument;         /* bit 0: count node visits / leaf tests (counting kernel variant);
                                   bit 1: time every trace, shade and guide launch with CUDA events on the
                                   context stream */
    int32_t samples_per_wave;   /* samples traced together in one wave (counter-based RNG only; the XORWOW
                                   states advance sample by sample): 0 = automatic (up to 16, at most about
                                   32M paths per wave), 1 = one sample per wave. Images do not depend on it:
                                   each pixel adds its samples in sample order. */
    int32_t env_sampling;       /* MC_ENV_SAMPLE_*: how next-event estimation picks environment directions */
    int32_t stack_entries;      /* traversal stack entries per lane: 0 = 64 (the reference's
                                   TRAVERSAL_STACK_CAPACITY, PT:1038); 1..63 shrink the trace kernel's
                                   shared memory; a ray that needs more ends and the call returns
                                   MC_ERR_STACK_OVERFLOW (builds keep every 4-wide tree within 64) */
    int32_t trace_threads;      /* trace block size: 256, or 128 (7 resident blocks per SM when the stack's
                                   shared memory allows; launches without density grids, reference
                                   intersector; other launches keep 256). 0 with stack_entries 0: 128 with
                                   the stack the 4-wide trees can need (3 entries per level) when that is at
                                   most 56, else 256. Images do not depend on it */
} mc_render_params;

enum {
    MC_ENV_SAMPLE_CDF = 0,      /* the reference's row/column CDF inversion (PT:433-467): four draws, two
                                   binary searches; image parity with the reference needs this mode */
    MC_ENV_SAMPLE_ALIAS = 1     /* Walker/Vose alias table over the texels (built by mc_env_create): four
                                   draws, one table read; the same texel distribution, so the same expected
                                   image, but not draw-compatible with the CDF mode */
};

#define MC_MAX_DEPTH 65536
#define MC_MAX_DEPTH_STATS 64
typedef struct mc_render_stats {
    int64_t extend_rays;        /* sum over bounces of extend-queue sizes */
    int64_t shadow_rays;        /* sum over bounces of shadow-queue sizes */
    int64_t paths;              /* width*height*spp */
    int64_t extend_per_depth[MC_MAX_DEPTH_STATS];   /* the last entry: depth 63 and deeper */
    int64_t shadow_per_depth[MC_MAX_DEPTH_STATS];
    int64_t node_visits;        /* traversal steps (instrument bit 0) */
    int64_t leaf_tests;         /* primitive intersection tests (instrument bit 0) */
    float render_ms;            /* device time of the sample loop (CUDA events) */
    float trace_ms;             /* summed device time of the trace launches (instrument bit 1) */
    int32_t trace_launches;     /* trace launches timed */
    int32_t kernel_launches;    /* library kernels launched by the call */
    int32_t error_flags;        /* device error word (MC_ERR_* bits) */
    float shade_ms;             /* summed device time of the shade launches (instrument bit 1) */
    float guide_infer_ms;       /* guided renders: guide inference launches (instrument bit 1) */
    float guide_train_ms;       /* guided renders: record compaction and Adam steps (instrument bit 1) */
} mc_render_stats;

/* ------------------------------------------------------------------------- */
/* Library, context, errors.                                                   */
/* ------------------------------------------------------------------------- */
MC_API const char* mc_version(void);
MC_API const char* mc_status_string(mc_status s);
/* Message of the last failed call on this host thread ("" if none). */
MC_API const char* mc_last_error(void);

/* A context owns the reusable wave buffers (path state, queues, RNG states) of
 * one device and one stream. One host thread at a time per context.
 * Replaces the per-call allocation in renderWithWavefront (PT:3757-3840). */
MC_API mc_status mc_context_create(int device, mc_context** out);
MC_API mc_status mc_context_destroy(mc_context* ctx);
/* Stream (cudaStream_t) all work of this context is issued on; NULL = legacy default. */
MC_API mc_status mc_context_set_stream(mc_context* ctx, void* stream);
/* Waits for the context's stream; returns MC_ERR_TIMEOUT (and clears it) when a
 * wait enqueued by mc_stream_wait_value ran out since the last call. */
MC_API mc_status mc_context_synchronize(mc_context* ctx);
/* Limit of the context's bounded device waits on an external flag
 * (mc_stream_wait_value), in microseconds; 0 restores the default of 2 s. */
MC_API mc_status mc_context_set_wait_timeout(mc_context* ctx, int64_t microseconds);
/* Makes the context's stream wait, on the device, until *d_flag >= value: a
 * 32-bit flag in device memory or mapped host memory that a producer outside
 * this stream sets (the host, another stream, a peer GPU). Unlike an unbounded
 * stream wait, the wait gives up after the context's wait timeout instead of
 * holding the GPU: work behind it then runs, and the next
 * mc_context_synchronize returns MC_ERR_TIMEOUT. The reference has no
 * counterpart (it synchronises the whole device after every launch,
 * PT:65-69). Returns once the wait is enqueued. */
MC_API mc_status mc_stream_wait_value(mc_context* ctx, const uint32_t* d_flag, uint32_t value);

/* ------------------------------------------------------------------------- */
/* Scene helpers (host).                                                       */
/* ------------------------------------------------------------------------- */
/* Camera::initialize (PT:1610-1631). */
MC_API mc_status mc_camera_initialize(mc_camera* cam);
/* triangle::calculate_bounding_box (PT:651-655) for every triangle, then the
 * emissive-triangle light list of finalizeScene (PT:1972-1985). lights may be
 * NULL to only count; *light_count receives the count. Host arrays. */
MC_API mc_status mc_scene_finalize_host(mc_triangle* tris, int32_t n, mc_light* lights, int32_t* light_count);
/* Splits host triangles into hot/cold records (PT:4276-4281). Host arrays. */
MC_API mc_status mc_split_triangles_host(const mc_triangle* tris, int32_t n, mc_triangle_hot* hot, mc_triangle_cold* cold);
/* Scene ingestion on the device: the triangle bounds and emissive-triangle
 * light list of finalizeScene (PT:1930-1987) and main()'s hot/cold split
 * (PT:4276-4289) as kernels, byte-identical to mc_scene_finalize_host followed
 * by mc_split_triangles_host. tris (n AoS records), hot and cold are device
 * arrays, 16-byte aligned; tris is not modified. lights: device array with
 * room for every emissive triangle (n is always enough), or NULL to only count.
 * spheres (device, n_sph records, may be NULL when n_sph is 0) are scanned for
 * media. light_count and has_medium (MC_MEDIUM_ANY when a primitive has a
 * material of type MC_MAT_ISOTROPIC, | MC_MEDIUM_GRID when one of those has a
 * density grid) are host outputs and may be NULL; the call synchronizes the
 * context's stream to read them. */
MC_API mc_status mc_scene_ingest(mc_context* ctx, const mc_triangle* tris, int32_t n, const mc_sphere* spheres,
                                 int32_t n_sph, mc_triangle_hot* hot, mc_triangle_cold* cold, mc_light* lights,
                                 int32_t* light_count, int32_t* has_medium);
/* mc_scene_ingest from a HOST array of AoS triangles (pageable or pinned):
 * uploads it (large pageable arrays through pinned staging filled by several
 * host threads), then ingests on the device. Other arguments as above. */
MC_API mc_status mc_scene_ingest_host(mc_context* ctx, const mc_triangle* tris, int32_t n, const mc_sphere* spheres,
                                      int32_t n_sph, mc_triangle_hot* hot, mc_triangle_cold* cold, mc_light* lights,
                                      int32_t* light_count, int32_t* has_medium);

/* Environment map from a host float RGBA image (top row first), with the
 * sampling tables of buildEnvironmentSamplingTables (PT:370-385). Creates the
 * device texture and tables; mc_env_destroy releases them. */
MC_API mc_status mc_env_create(const float* rgba_host, int32_t width, int32_t height, float intensity,
                               float rotation_radians, mc_env_map* out);
MC_API mc_status mc_env_destroy(mc_env_map* env);

/* ------------------------------------------------------------------------- */
/* Heterogeneous media (PT:784-838). An isotropic material whose density_grid  */
/* is set scatters by delta tracking and attenuates shadow rays by ratio       */
/* tracking, with extinction density x grid value and majorant density x      */
/* grid_max_density; without a grid it stays homogeneous (PT:3559-3566).       */
/* ------------------------------------------------------------------------- */
/* The reference's grid is a NanoVDB FloatGrid (openvdb v12.0.1, nanovdb/
 * subtree, not vendored), read through its world-to-index map and a
 * trilinear sampler (PT:784-789). This grid is dense: FP32 voxels, x fastest,
 * voxel (i,j,k) centred at origin + voxel_size * (i,j,k), value 0 outside.
 * Index coordinates are (p - origin) * inv_voxel_size; the sample at index
 * point x interpolates the 8 voxels around floor(x), z first, then y, then x,
 * each step a + w * (b - a) as one fused multiply-add. The device copy is
 * self-contained: this 64-byte header, then the voxels. */
typedef struct mc_volume_grid {
    MC_ALIGNAS(16) float origin[3];
    float voxel_size;
    float inv_voxel_size;
    int32_t dims[3];
    float maximum_density;      /* largest voxel value: the majorant (root().maximum() in NanoVDB) */
    float world_min[3];         /* centre of voxel (0,0,0) */
    float world_max[3];         /* centre of the last voxel */
    int32_t pad0;
} mc_volume_grid;

enum {
    MC_MEDIUM_ANY = 1,          /* mc_scene_view.has_medium bits: an isotropic material (PT:4328-4331) */
    MC_MEDIUM_GRID = 2          /* ... of which at least one carries a density grid */
};

/* Copies nx*ny*nz host densities (x fastest; finite, >= 0) to a device grid.
 * *d_grid receives the device pointer that mc_material.density_grid takes;
 * *header (optional) the header, whose maximum_density goes into
 * mc_material.grid_max_density. mc_volume_grid_destroy frees it. */
MC_API mc_status mc_volume_grid_create(mc_context* ctx, const float* density_host, int32_t nx, int32_t ny, int32_t nz,
                                       const float origin[3], float voxel_size, const mc_volume_grid** d_grid,
                                       mc_volume_grid* header);
MC_API mc_status mc_volume_grid_destroy(const mc_volume_grid* d_grid);
/* The fog sphere of createFogSphereGrid (src/volume_io.cpp:53-64, nanovdb's
 * createFogVolumeSphere) centred at the origin: a narrow band of half_width
 * voxels (nanovdb's default 3) inside the surface ramps the density linearly
 * from 0 at the surface to 1, the interior is 1, the outside 0. Voxel values
 * are clamp((radius - |p|) / (half_width * voxel_size), 0, 1) at the voxel
 * centres p, computed in double. The grid spans ceil(radius / voxel_size) + 1
 * voxels on each side of the centre voxel. With density_host NULL only dims
 * and origin are returned. */
MC_API mc_status mc_volume_fog_sphere(float radius, float voxel_size, float half_width, float* density_host,
                                      int32_t dims[3], float origin[3]);
/* A dense grid file (the --volume file of the command-line driver): one
 * text line "MCVOL nx ny nz voxel_size origin_x origin_y origin_z" and a
 * newline, then nx*ny*nz little-endian float32 densities, x fastest.
 * density_host NULL only reads the header. */
MC_API mc_status mc_volume_file_read(const char* path, int32_t dims[3], float origin[3], float* voxel_size,
                                     float* density_host);
MC_API mc_status mc_volume_file_write(const char* path, const int32_t dims[3], const float origin[3], float voxel_size,
                                      const float* density_host);
/* Grid values at n world points (device, xyz packed) as the media sample them. */
MC_API mc_status mc_volume_density(mc_context* ctx, const mc_volume_grid* d_grid, const float* d_points, int32_t n,
                                   float* d_out);

/* ------------------------------------------------------------------------- */
/* Synthetic scenes (seeded, deterministic). Host output.                      */
/* ------------------------------------------------------------------------- */
enum {
    MC_SCENE_CORNELL_BOXES = 1,      /* Cornell room, white floor, two rotated boxes (36 triangles) */
    MC_SCENE_DISPLACED_ICOSPHERES = 2, /* 3 displaced level-L icospheres + ground + medium box + light + sky */
    MC_SCENE_BATCH_MEMBER = 3,       /* one scene of the 64-scene batch (index = variant) */
    MC_SCENE_GUIDING_ROOM = 4,       /* 10x10x4 room lit through a 0.2x0.2 aperture */
    MC_SCENE_CORNELL_SPHERES = 5     /* the reference's buildCornellScene (spheres, medium, motion) minus the image texture */
};

typedef struct mc_scene_desc {
    int32_t kind;                /* MC_SCENE_* */
    int32_t variant;             /* batch member index / icosphere subdivision level (0 = default) */
    uint64_t seed;
    int32_t triangle_target;     /* batch members: requested triangle count (0 = drawn from the seed) */
} mc_scene_desc;

typedef struct mc_scene_host {
    mc_triangle* triangles;  int32_t triangle_count;
    mc_sphere* spheres;      int32_t sphere_count;
    mc_camera camera;            /* initialized for the scene's default resolution */
    int32_t width, height, spp, max_depth;
    int32_t has_medium;
    float* env_rgba;             /* NULL or env_width*env_height*4 floats, top row first */
    int32_t env_width, env_height;
    float env_intensity;
} mc_scene_host;

MC_API mc_status mc_scene_generate(const mc_scene_desc* desc, mc_scene_host* out);
/* The reference's cloud scene (buildCloudScene PT:1849-1891 and main()'s
 * cloud camera PT:4148-4167) around a density grid: an isotropic sphere
 * enclosing the grid's bounds (albedo 1, density scale 4, g 0.877, carrying
 * d_grid and header->maximum_density), a ground quad 1000 below, and with
 * sun != 0 (the reference's choice without --env) a far emissive quad in
 * the sun's direction; 333x180, 500 spp, max depth 1000, roulette cap 0.95,
 * the Mitsuba sensor. d_grid: from mc_volume_grid_create; header: its header. */
MC_API mc_status mc_scene_cloud(const mc_volume_grid* d_grid, const mc_volume_grid* header, int32_t sun,
                                mc_scene_host* out);
MC_API mc_status mc_scene_free(mc_scene_host* scene);

/* OBJ/MTL loading: loadObject (PT:2644-2859) with loadMtlFile (PT:2614-2680).
 * Appends the file's triangles to scene->triangles (reallocated; free with
 * mc_scene_free). The model is centred on x/z with its lowest point at y = 0
 * and its largest side 1, then scaled by `scale`, rotated by rotation_y
 * radians about y and moved by `translation`. Faces are fan-triangulated;
 * faces with a bad index or zero area are skipped; without vn the normals are
 * area-weighted vertex averages. Materials: newmtl/Kd/Ke/map_Kd, emissive when
 * Ke has a positive component, else lambertian (with the map_Kd image read
 * from a .ppm beside the named file when load_textures is set and it loads);
 * faces without a known material get *fallback. Errors: MC_ERR_NOT_FOUND (no
 * such file), MC_ERR_INVALID (no vertices, faces or triangles). */
typedef struct mc_obj_info {
    int32_t triangles_added;
    int32_t faces_skipped;
    int32_t materials;
    int32_t textures_loaded;
    int32_t textures_missing;   /* materials whose map_Kd image was not loaded */
    int32_t unknown_materials;  /* usemtl names the libraries do not define */
    uint64_t* textures;         /* the textures_loaded textures created (mc_image_texture_destroy each,
                                   then mc_obj_info_free) */
} mc_obj_info;
MC_API mc_status mc_obj_load(const char* path, const mc_material* fallback, mc_vec3 translation, float scale,
                             float rotation_y, int32_t load_textures, mc_scene_host* scene, mc_obj_info* info);
MC_API mc_status mc_obj_info_free(mc_obj_info* info);
/* loadPpmAsRgba8 (PT:236-294): a binary PPM (P6, maximum 255) as RGBA8 with
 * alpha 255. rgba NULL only reads the size. */
MC_API mc_status mc_ppm_read(const char* path, int32_t* width, int32_t* height, uint8_t* rgba);
/* loadPfmAsRgba32f (PT:335-368): a little-endian colour PFM ("PF", negative
 * scale) as float RGBA, top row first, alpha 1; the environment maps of
 * --env. The header's four fields are whitespace-separated and exactly one
 * byte follows them. rgba NULL only reads the size. */
MC_API mc_status mc_pfm_read(const char* path, int32_t* width, int32_t* height, float* rgba);
/* createImageTextureObject (PT:296-316): an RGBA8 image texture (sRGB,
 * bilinear, wrapped) for mc_texture.image; mc_image_texture_destroy frees it. */
MC_API mc_status mc_image_texture_create(const uint8_t* rgba, int32_t width, int32_t height, uint64_t* texture);
MC_API mc_status mc_image_texture_destroy(uint64_t texture);

/* ------------------------------------------------------------------------- */
/* BVH (a1-a7). Replaces the host Morton/sort (PT:1930-1987, 4223-4260) and    */
/* BVH::generateHierarchy (PT:1063-1090).                                      */
/* ------------------------------------------------------------------------- */
/* Morton codes of the reference's primitive list (spheres first, then
 * triangles; PT:1955-1971) in the scene's bounds. d_codes: device, n entries.
 * *bounds_out (host, may be NULL) receives the scene bounds. */
MC_API mc_status mc_morton_codes(mc_context* ctx, const mc_scene_view* scene, uint32_t* d_codes, mc_aabb* bounds_out);

/* Stable LSD radix sort of 30-bit keys with their values (onesweep-style,
 * 4 passes of 8 bits). Device arrays; in place through context scratch. */
MC_API mc_status mc_radix_sort_pairs(mc_context* ctx, uint32_t* d_keys, int32_t* d_values, int32_t n, int32_t key_bits);

/* Largest n that mc_radix_sort_pairs_static accepts. */
#define MC_SORT_STATIC_MAX_PAIRS (1 << 20)

/* The same stable radix sort as mc_radix_sort_pairs, with the same results,
 * for callers that must not allocate device memory when they sort. This entry
 * point has no counterpart in the reference (whose sort is a host std::sort).
 *
 * Who needs it: a caller whose device memory is fully handed out ahead of time
 * (a render server that admits jobs up to a fixed HBM budget has nothing left
 * to allocate from at request time) and a caller whose memory belongs to
 * another allocator (a caching allocator such as PyTorch's, which a direct
 * cudaMalloc would bypass and fragment). This call allocates nothing: no
 * cudaMalloc/cudaFree and no allocating library routine.
 *
 * Synchronisation: a call with n > 1 waits for ctx's stream to finish before
 * it returns (it reads the device error word written by the sort's bounded
 * waits), like mc_radix_sort_pairs.
 *
 * Scratch: a fixed device array inside the library (about 9 MiB: the
 * alternate key/value arrays for MC_SORT_STATIC_MAX_PAIRS pairs, the digit
 * histograms, tile counters and look-back status), one per device, reserved
 * when the library's device code loads. n > MC_SORT_STATIC_MAX_PAIRS returns
 * MC_ERR_INVALID without touching the arrays; sort larger arrays with
 * mc_radix_sort_pairs. The histograms, counters and status words are cleared
 * on ctx's stream by every call.
 *
 * Set-up: the first call on a device looks up that device's scratch address
 * (with the device made current for the look-up) and loads the sort kernels.
 * Make that first call before any stream capture begins: a call with n = 0
 * (keys and values may be NULL) does the set-up and nothing else.
 *
 * Overlapping calls race: every call on one device shares the one scratch
 * array, so two calls whose work overlaps in time (from two threads, or on two
 * streams) corrupt each other's results. Issue them one after another, on one
 * stream or with the earlier one finished. */
MC_API mc_status mc_radix_sort_pairs_static(mc_context* ctx, uint32_t* d_keys, int32_t* d_values, int32_t n,
                                            int32_t key_bits);

/* Full build: bounds, Morton codes, sort, Karras hierarchy, refit, layout. */
MC_API mc_status mc_bvh_build(mc_context* ctx, const mc_scene_view* scene, const mc_bvh_build_opts* opts, mc_bvh** out);
/* One build over `count` scenes in a single pass of launches: per-scene bounds
 * and Morton codes, one stable sort by (scene, code), per-scene Karras trees,
 * refit and collapse. The handle holds every scene's tree (scene i = the i-th
 * view); render it with mc_render_batch. Each scene needs >= 2 primitives. */
MC_API mc_status mc_bvh_build_batch(mc_context* ctx, const mc_scene_view* scenes, int32_t count,
                                    const mc_bvh_build_opts* opts, mc_bvh** out);
/* A tree's buffers and a build's temporaries come from a stream-ordered pool
 * of the device that keeps freed memory for the next build (the process's
 * pools outlive contexts; mc_context_destroy hands back what they hold
 * unused). mc_bvh_free waits for the device's work, as cudaFree would, and
 * may be called after the building context is destroyed. */
MC_API mc_status mc_bvh_free(mc_bvh* bvh);
MC_API mc_status mc_bvh_get_info(const mc_bvh* bvh, mc_bvh_info* info);
/* Export in the reference's representation (device arrays, any may be NULL):
 * sorted codes / primitive ids / primitive types (n each), internal nodes
 * (n-1) and leaves (n) as mc_bvh_node. Needs keep_reference_nodes for nodes. */
MC_API mc_status mc_bvh_export(const mc_bvh* bvh, uint32_t* d_codes, int32_t* d_ids, int32_t* d_types,
                               mc_bvh_node* d_internal, mc_bvh_node* d_leaves);
/* Copies of the arrays the traversal reads (device buffers, either may be
 * NULL): the node array (mc_bvh_info.node_bytes bytes) and the leaf-ordered
 * primitive records (mc_bvh_info.prim_bytes bytes), e.g. to store a built tree
 * or to compare two builds byte for byte. No counterpart in the reference,
 * whose traversal reads its exported node layout directly. */
MC_API mc_status mc_bvh_export_traversal(const mc_bvh* bvh, void* d_nodes, void* d_prims);

/* ------------------------------------------------------------------------- */
/* Ray sets (a8-a15). Rays are SoA: 7 device float arrays of n entries packed  */
/* back to back: ox[n], oy[n], oz[n], dx[n], dy[n], dz[n], time[n].            */
/* ------------------------------------------------------------------------- */
/* Closest hit per ray, as extendKernelPersistent writes it (PT:3402-3468). */
MC_API mc_status mc_trace_closest(mc_context* ctx, const mc_bvh* bvh, const mc_scene_view* scene,
                                  const float* d_rays, int32_t n, int32_t intersector, mc_packed_hit* d_hits);
/* Any hit within (1e-4, tmax) per ray, as traverseAnyHit (PT:1152-1207).
 * d_occluded[i] = 1 when blocked. */
MC_API mc_status mc_trace_any(mc_context* ctx, const mc_bvh* bvh, const mc_scene_view* scene,
                              const float* d_rays, const float* d_tmax, int32_t n, int32_t intersector,
                              int32_t* d_occluded);

/* ------------------------------------------------------------------------- */
/* Rendering (a16-a22). Replaces renderWithWavefront (PT:3757-3840).          */
/* d_accum: device float3 per pixel (W*H*12 bytes, row-major, y=0 top), the   */
/* reference's linear accumulation buffer; samples are added to it.            */
/* ------------------------------------------------------------------------- */
MC_API mc_status mc_render_wavefront(mc_context* ctx, const mc_bvh* bvh, const mc_scene_view* scene,
                                     const mc_render_params* params, float* d_accum, mc_render_stats* stats);
/* One scene of a batched render. */
typedef struct mc_batch_item {
    mc_scene_view scene;        /* device arrays of this scene */
    mc_render_params params;    /* camera, size, spp, first_sample, max depth, seed (counter-based RNG) */
    float* d_accum;             /* this scene's accumulation buffer (W*H float3) */
} mc_batch_item;

/* Renders every item of a batch BVH (mc_bvh_build_batch, same scene order) in
 * shared waves: each wave holds one sample of every pixel of every item that
 * still needs samples, traced and shaded by the same persistent launches.
 * use_graph: capture the wave's launch sequence once as a CUDA graph and
 * replay it per wave. Layout, persistence and intersector come from items[0]. */
MC_API mc_status mc_render_batch(mc_context* ctx, const mc_bvh* bvh, const mc_batch_item* items, int32_t count,
                                 int32_t use_graph, mc_render_stats* stats);

/* Same call with host memory: copies the scene in, builds, renders, copies the
 * accumulation buffer out (accum_host: W*H*3 floats, accumulated into). */
MC_API mc_status mc_render_host(mc_context* ctx, const mc_triangle* tris, int32_t n_tri,
                                const mc_sphere* spheres, int32_t n_sph, const mc_env_map* env,
                                const mc_render_params* params, float* accum_host, mc_render_stats* stats);
/* Reset the per-pixel XORWOW states (PT:2865-2871 init_rng_kernel). */
MC_API mc_status mc_rng_reset(mc_context* ctx, int32_t width, int32_t height, uint64_t seed);

/* Sets params' launch configuration to the fastest found by timing real
 * waves of this render on this scene and BVH: the trace variant (persistent
 * or plain) and refill_threshold; the trace block shape (trace_threads 256,
 * or 128 with stack_entries cut to what the 4-wide tree can need, 3 per
 * level, when that lets 7 blocks share an SM); the queue capacity, as
 * samples_per_wave (a wave's queues hold width x height x samples_per_wave
 * entries: the automatic choice, or twice it while spp and about 64M paths
 * allow; compared per sample); and use_graph. Cached per (device, layout,
 * scene size class, image size class, spp class); the image does not depend
 * on any choice. budget_ms bounds the tuning time (0 = 2000). */
MC_API mc_status mc_autotune(mc_context* ctx, const mc_bvh* bvh, const mc_scene_view* scene,
                             mc_render_params* params, int32_t budget_ms);

/* ------------------------------------------------------------------------- */
/* Learned path guiding. No counterpart in the reference: its shade kernel    */
/* samples the BSDF only (PT:3645-3690).                                      */
/*                                                                           */
/* A small MLP maps an encoded (position, ray direction) to a mixture of 8   */
/* von Mises-Fisher lobes over the next direction. Input: each of the 6      */
/* coordinates (position normalized to the guide's box, direction) encoded   */
/* as sin/cos(pi * 2^f * x), f = 0..11 (144 inputs); three hidden layers of  */
/* 64 ReLU units; 40 outputs (8 logits, 8 x 3 unnormalized means, 8 log      */
/* concentrations). BF16 weights and activations, FP32 accumulation on the   */
/* tensor cores (tcgen05), FP32 master weights updated by Adam.              */
/* ------------------------------------------------------------------------- */
#define MC_GUIDE_INPUTS 144
#define MC_GUIDE_HIDDEN 64
#define MC_GUIDE_LOBES 8
#define MC_GUIDE_OUTPUTS 40
/* Flat FP32 parameter vector: W1[64][144] b1[64] W2[64][64] b2[64] W3[64][64]
 * b3[64] W4[40][64] b4[40] (W[out][in], row-major). */
#define MC_GUIDE_PARAM_COUNT 20200
/* Per query: x, y, z, dx, dy, dz (world position, the direction input: a
 * unit normal or ray direction, mc_guide_config.direction_input). */
#define MC_GUIDE_QUERY_FLOATS 6
/* Per training record: position, the direction input at the vertex, the
 * sampled next direction, and the record's weight (the radiance estimate
 * carried back through that direction divided by its sampling density, a
 * luminance). */
#define MC_GUIDE_RECORD_FLOATS 10
/* Per query output: lobe weights[8] (sum 1), unit means[8][3], kappa[8]. */
#define MC_GUIDE_MIXTURE_FLOATS 40

typedef struct mc_guide mc_guide;

typedef struct mc_guide_config {
    mc_aabb bounds;             /* positions are normalized to this box */
    float learning_rate;        /* Adam; 0 = 1e-3 */
    float beta1, beta2, epsilon;/* 0 = 0.9, 0.999, 1e-8 */
    uint64_t seed;              /* weight initialization */
    int32_t batch_capacity;     /* records per training step in guided renders; 0 = 65536 */
    float guide_fraction;       /* one-sample MIS mix: probability of sampling the guide; 0 = 0.5 */
    int32_t train_steps;        /* Adam steps per sample in guided renders, each on its own
                                   batch_capacity records of that sample; 0 = 1 */
    int32_t train_vertices;     /* guided renders: diffuse vertices per path that give training records,
                                   the first ones along the path (1..MC_GUIDE_MAX_TRAIN_VERTICES); 0 = 1 */
    int32_t direction_input;    /* MC_GUIDE_DIR_*: the direction the guided renderer feeds the network */
    int32_t guided_depth;       /* guided renders: bounces whose diffuse vertices sample the guide (the network
                                   runs only for those); deeper vertices sample the cosine lobe alone. 0 = 2
                                   (the first bounce); never below train_vertices + 1 when training;
                                   MC_MAX_DEPTH = every bounce */
    float weight_cap;           /* guided renders' training: a record's share of its step's normalized weight
                                   is capped at weight_cap / (records in the step), so a few rare bright paths
                                   cannot take over a step (0 = no cap). The estimator stays unbiased: only
                                   the proposal the guide learns changes */
    int32_t fold_below;         /* guided renders: the guide's directions below the surface are mirrored up
                                   (the density counts both) instead of ending the path; 0 = off */
    int32_t anchor_lobes;       /* MC_GUIDE_LOBES_*. Anchored (the default): every lobe's mean is the
                                   network's raw mean output plus MC_GUIDE_ANCHOR times the direction input
                                   (turned away from the surface for MC_GUIDE_DIR_RAY), normalized, and kappa
                                   starts near e: an untrained guide proposes directions around the normal, a
                                   cosine-like lobe, instead of a near-uniform sphere whose lower half ends
                                   paths. Raw: the means are the raw outputs, normalized */
    int32_t nee_records;        /* 1: guided renders' training also takes a record from each primary diffuse
                                   vertex's next-event sample (the direction to the light point, weighted by
                                   the light it brought, times its MIS weight), and the records of that vertex's
                                   sampled direction keep only their MIS-weighted share of the emission they
                                   found: the two kinds together still estimate the incident light, and every
                                   unoccluded shadow ray toward a small light becomes a training sample.
                                   0 = off */
} mc_guide_config;

/* Length of the direction-input offset added to every raw lobe mean of an
 * anchored guide. */
#define MC_GUIDE_ANCHOR 1.5f
enum {
    MC_GUIDE_LOBES_DEFAULT = 0, /* anchored */
    MC_GUIDE_LOBES_ANCHORED = 1,
    MC_GUIDE_LOBES_RAW = 2
};

#define MC_GUIDE_MAX_TRAIN_VERTICES 4
enum {
    MC_GUIDE_DIR_NORMAL = 0,    /* the vertex's geometric normal, turned to face the arriving ray: the
                                   incident light of a diffuse vertex depends on where it is and which way
                                   it faces, not on the direction it is seen from */
    MC_GUIDE_DIR_RAY = 1        /* the arriving ray's direction */
};

MC_API mc_status mc_guide_create(mc_context* ctx, const mc_guide_config* config, mc_guide** out);
MC_API mc_status mc_guide_destroy(mc_guide* guide);
/* FP32 master parameters (host arrays of MC_GUIDE_PARAM_COUNT floats). */
MC_API mc_status mc_guide_get_params(const mc_guide* guide, float* params);
MC_API mc_status mc_guide_set_params(mc_guide* guide, const float* params);
/* Mixtures for n queries (device arrays). */
MC_API mc_status mc_guide_infer(mc_guide* guide, const float* d_queries, int32_t n, float* d_mixtures);
/* Gradient of sum_i weight_i * -log q(next_i | position_i, direction_i) over
 * n records, w.r.t. the flat parameters (d_grad: device, PARAM_COUNT floats);
 * *loss (host, may be NULL) receives the loss. No parameter update. */
MC_API mc_status mc_guide_gradient(mc_guide* guide, const float* d_records, int32_t n, float* d_grad, double* loss);
/* One Adam step on n records, with the weights normalized to sum 1. */
MC_API mc_status mc_guide_train(mc_guide* guide, const float* d_records, int32_t n);
/* Adam steps taken so far. */
MC_API int32_t mc_guide_steps(const mc_guide* guide);

/* Guided wavefront render: at diffuse vertices the next direction comes from
 * the guide with probability guide_fraction and from the cosine BSDF
 * otherwise, weighted by the mixed density (one-sample MIS, unbiased); NEE's
 * MIS weights use the same mixed density. With train != 0 the first
 * train_vertices diffuse vertices of every path become training records
 * (weight: the light that arrived through the sampled direction, excluding
 * the vertex's own NEE, over the throughput that reached the vertex and the
 * direction's density) and the guide takes train_steps Adam steps per sample.
 * Needs the counter-based RNG and a single-scene BVH. */
MC_API mc_status mc_render_guided(mc_context* ctx, const mc_bvh* bvh, const mc_scene_view* scene,
                                  const mc_render_params* params, mc_guide* guide, int32_t train, float* d_accum,
                                  mc_render_stats* stats);

/* ------------------------------------------------------------------------- */
/* Resolve and output encoding.                                                */
/* ------------------------------------------------------------------------- */
/* PT:3073 ToneMapOption */
enum { MC_TONEMAP_NONE = 0, MC_TONEMAP_REINHARD = 1, MC_TONEMAP_ACES = 2 };
enum {
    MC_IMAGE_RGB8 = 0,      /* W*H*3 bytes, top row first: the pixels main() writes to the PNG (PT:4363-4380) */
    MC_IMAGE_RGB_F32 = 1,   /* W*H float3: resolve_kernel's frame buffer (PT:3092-3100), sRGB-encoded */
    MC_IMAGE_PFM = 2,       /* a little-endian PFM file: "PF\n<W> <H>\n-1.0\n" and W*H float3 of linear
                               radiance (average x exposure, no tone map), bottom row first */
    MC_IMAGE_PNG = 3        /* a PNG file of the MC_IMAGE_RGB8 pixels (stored deflate blocks) */
};
typedef struct mc_image_options {
    int32_t format;         /* MC_IMAGE_* */
    int32_t tonemap;        /* MC_TONEMAP_* (RGB8, RGB_F32, PNG) */
    float exposure;         /* > 0: multiplier; <= 0: automatic, computeAutoExposure (PT:3121-3132) */
    int32_t device_output;  /* 1: out is device memory (RGB8 and RGB_F32 only) */
} mc_image_options;

/* Resolves an accumulation buffer once (the reference resolves after every
 * sample, PT:3823) and encodes it: average over `samples`, exposure, tone map,
 * sRGB, 8-bit quantisation with main()'s NaN shield, in one pass over the
 * buffer. accum: device, W*H float3. out: host memory (or device memory with
 * opts.device_output, RGB8 and RGB_F32 only) of at least *bytes; out NULL only reports the size in
 * *bytes. chosen_exposure (host, may be NULL): the exposure applied. An
 * automatic exposure sums ln(1e-4 + luminance) in a fixed order in FP64 (the
 * reference adds FP32 warp sums with atomics, in no fixed order). */
MC_API mc_status mc_image_encode(mc_context* ctx, const float* accum, int32_t width, int32_t height, int32_t samples,
                                 const mc_image_options* opts, void* out, int64_t* bytes, float* chosen_exposure);
/* mc_image_encode of a HOST accumulation buffer (uploaded first); out is host
 * memory. */
MC_API mc_status mc_image_encode_host(mc_context* ctx, const float* accum_host, int32_t width, int32_t height,
                                      int32_t samples, const mc_image_options* opts, void* out, int64_t* bytes,
                                      float* chosen_exposure);
/* Host: a PNG file (8-bit RGB, no interlace, stored deflate blocks) of
 * W*H*3 bytes of pixels, top row first. out NULL only reports *bytes. */
MC_API mc_status mc_png_encode(const uint8_t* rgb, int32_t width, int32_t height, uint8_t* out, int64_t* bytes);

/* ------------------------------------------------------------------------- */
/* Render server. No counterpart in the reference (one scene per process).   */
/*                                                                           */
/* Scenes are registered once; their BVHs stay resident. Requests (scene,    */
/* camera, size, spp, seed, guided or not) are admitted in arrival order     */
/* while their memory fits the HBM budget (accumulation buffer, their share  */
/* of the wave buffers and, for guided requests, the guide's per-path        */
/* buffers); a request that could never fit is refused with MC_ERR_BUDGET.   */
/* Each mc_server_step renders samples_per_step samples of the active        */
/* requests it schedules (the oldest, then least remaining work first, up to */
/* wave_paths paths): the plain ones of all scenes share the same waves (one */
/* persistent trace launch and one shade launch per bounce for all of them), */
/* guided ones run their scene's guided render. A request is done when it    */
/* has all its samples; its accumulation buffer stays until released.        */
/* Times are host seconds since the server was created.                      */
/* ------------------------------------------------------------------------- */
typedef struct mc_server mc_server;

typedef struct mc_server_config {
    int64_t hbm_budget_bytes;   /* 0 = 150 GB */
    int32_t max_active;         /* requests admitted at a time (<= 128); 0 = 128 */
    int32_t samples_per_step;   /* 0 = 16 (traced in one wave per step for plain requests) */
    int64_t wave_paths;         /* paths a step renders per sample: the oldest active request,
                                   then the ones with the least remaining work while they fit;
                                   0 = 4194304 */
    int32_t flags;              /* MC_SERVER_* */
    int32_t pad0;
} mc_server_config;

/* A step renders the plain requests of each scene in a wave of their own
 * (single-scene trace launches) instead of one wave shared by every scene. */
#define MC_SERVER_SCENE_WAVES 1

typedef struct mc_server_request {
    int64_t scene_id;
    mc_render_params params;    /* camera, size, spp, seed, max depth (counter-based RNG) */
    int32_t guided;             /* render with the scene's guide (trained online) */
} mc_server_request;

enum { MC_REQ_PENDING = 0, MC_REQ_ACTIVE = 1, MC_REQ_DONE = 2, MC_REQ_RELEASED = 3, MC_REQ_CANCELLED = 4 };

typedef struct mc_server_result {
    int64_t request_id;
    int32_t state;              /* MC_REQ_* */
    int32_t spp_done;
    double submit_s, admit_s, done_s;
    int64_t bytes;              /* memory charged to the budget until released */
    const float* d_accum;       /* W*H float3 accumulation (valid until released) */
} mc_server_result;

typedef struct mc_server_stats {
    int64_t budget_bytes, used_bytes, scene_bytes;
    int32_t scenes, pending, active, done;
    int64_t steps, waves, rays;
} mc_server_stats;

MC_API mc_status mc_server_create(mc_context* ctx, const mc_server_config* config, mc_server** out);
MC_API mc_status mc_server_destroy(mc_server* server);
/* Builds the scene's 4-wide BVH; the scene arrays stay owned by the caller
 * and must outlive the server. *scene_id: the id requests refer to. */
MC_API mc_status mc_server_add_scene(mc_server* server, const mc_scene_view* scene, int64_t* scene_id);
MC_API mc_status mc_server_submit(mc_server* server, const mc_server_request* request, int64_t* request_id);
/* Admits what fits, renders one step, retires finished requests.
 * *active (may be NULL): requests active after the step. */
MC_API mc_status mc_server_step(mc_server* server, int32_t* active);
MC_API mc_status mc_server_get_result(mc_server* server, int64_t request_id, mc_server_result* result);
/* Copies a request's accumulation buffer (W*H float3, the sum over its
 * samples so far) into host memory. */
MC_API mc_status mc_server_read(mc_server* server, int64_t request_id, float* host_rgb);
/* Encodes a request's image as mc_image_encode does (samples = the samples
 * accumulated so far) into host memory; out NULL only reports *bytes. */
MC_API mc_status mc_server_encode(mc_server* server, int64_t request_id, const mc_image_options* opts, void* out,
                                  int64_t* bytes, float* chosen_exposure);
/* Frees a finished request's accumulation buffer. */
MC_API mc_status mc_server_release(mc_server* server, int64_t request_id);
/* Cancels a pending or active request between steps (a client that went away,
 * a deadline missed): it leaves the schedule, its accumulation buffer is freed
 * and its memory returns to the budget at once; its state becomes
 * MC_REQ_CANCELLED with the samples it had (spp_done). Reading or encoding it
 * afterwards returns MC_ERR_CANCELLED. The reference has no counterpart (its
 * only way out is exit(), PT:55-63). A request that is already done (or
 * released) is not cancelled: MC_ERR_INVALID. */
MC_API mc_status mc_server_cancel(mc_server* server, int64_t request_id);
MC_API mc_status mc_server_get_stats(const mc_server* server, mc_server_stats* stats);
/* Host seconds since the server was created (the clock of the results). */
MC_API double mc_server_now(const mc_server* server);

#ifdef __cplusplus
} /* extern "C" */
#endif

/* ------------------------------------------------------------------------- */
/* Layout pins (sizes measured on the reference compiled with nvcc 12.9).       */
/* ------------------------------------------------------------------------- */
#ifdef __cplusplus
#define MC_STATIC_ASSERT(c, m) static_assert(c, m)
#else
#define MC_STATIC_ASSERT(c, m) _Static_assert(c, m)
#endif
MC_STATIC_ASSERT(sizeof(mc_vec3) == 12, "vec3 is 12 bytes");
MC_STATIC_ASSERT(sizeof(mc_aabb) == 32, "AABB is 32 bytes");
MC_STATIC_ASSERT(sizeof(mc_texture) == 40, "Texture is 40 bytes");
MC_STATIC_ASSERT(sizeof(mc_material) == 96, "Material is 96 bytes");
MC_STATIC_ASSERT(sizeof(mc_triangle) == 224, "triangle is 224 bytes");
MC_STATIC_ASSERT(sizeof(mc_triangle_hot) == 36, "triangle_hot is 36 bytes");
MC_STATIC_ASSERT(sizeof(mc_triangle_cold) == 192, "triangle_cold is 192 bytes");
MC_STATIC_ASSERT(offsetof(mc_triangle_cold, mat) == 64, "triangle_cold.mat at 64");
MC_STATIC_ASSERT(offsetof(mc_triangle_cold, aabb) == 160, "triangle_cold.aabb at 160");
MC_STATIC_ASSERT(sizeof(mc_sphere) == 160, "sphere is 160 bytes");
MC_STATIC_ASSERT(offsetof(mc_sphere, mat) == 32, "sphere.mat at 32");
MC_STATIC_ASSERT(offsetof(mc_sphere, aabb) == 128, "sphere.aabb at 128");
MC_STATIC_ASSERT(sizeof(mc_light) == 64, "Light is 64 bytes");
MC_STATIC_ASSERT(sizeof(mc_bvh_node) == 64, "BVH_Node is 64 bytes");
MC_STATIC_ASSERT(offsetof(mc_bvh_node, left) == 32, "BVH_Node.leftChild at 32");
MC_STATIC_ASSERT(offsetof(mc_bvh_node, right) == 36, "BVH_Node.rightChild at 36");
MC_STATIC_ASSERT(offsetof(mc_bvh_node, left_is_leaf) == 40, "BVH_Node.leftIsLeaf at 40");
MC_STATIC_ASSERT(offsetof(mc_bvh_node, right_is_leaf) == 41, "BVH_Node.rightIsLeaf at 41");
MC_STATIC_ASSERT(offsetof(mc_bvh_node, parent) == 44, "BVH_Node.parent at 44");
MC_STATIC_ASSERT(offsetof(mc_bvh_node, prim) == 48, "BVH_Node.primitiveIndex at 48");
MC_STATIC_ASSERT(offsetof(mc_bvh_node, is_leaf) == 52, "BVH_Node.isLeaf at 52");
MC_STATIC_ASSERT(sizeof(mc_packed_hit) == 16, "PackedHit is 16 bytes");
MC_STATIC_ASSERT(sizeof(mc_camera) == 172, "Camera is 172 bytes");
MC_STATIC_ASSERT(sizeof(mc_env_map) == 56, "EnvironmentMap is 56 bytes");
/* this library's own structs (bindings mirror these sizes) */
MC_STATIC_ASSERT(sizeof(mc_guide_config) == 96, "mc_guide_config is 96 bytes");
MC_STATIC_ASSERT(sizeof(mc_render_params) == 248, "mc_render_params is 248 bytes");
MC_STATIC_ASSERT(sizeof(mc_server_config) == 32, "mc_server_config is 32 bytes");
MC_STATIC_ASSERT(sizeof(mc_server_request) == 264, "mc_server_request is 264 bytes");
MC_STATIC_ASSERT(sizeof(mc_server_result) == 56, "mc_server_result is 56 bytes");
MC_STATIC_ASSERT(sizeof(mc_server_stats) == 64, "mc_server_stats is 64 bytes");
MC_STATIC_ASSERT(sizeof(mc_image_options) == 16, "mc_image_options is 16 bytes");
MC_STATIC_ASSERT(sizeof(mc_obj_info) == 32, "mc_obj_info is 32 bytes");

#endif /* MC_ABI_H */
