// mc_internal.h - library-internal declarations shared by the .cu/.cpp files.
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>

#include "mc_abi.h"

#ifdef __CUDACC__
#include <cuda_runtime.h>
#else
typedef struct CUstream_st* cudaStream_t;
#endif

// Device error word bits (written with atomicOr by kernels, read by the host).
#define MC_DEVERR_STACK 1
#define MC_DEVERR_QUEUE 2
#define MC_DEVERR_TIMEOUT 4
#define MC_DEVERR_INPUT 8

// Traversal stack capacity (the reference's TRAVERSAL_STACK_CAPACITY, PT:1038).
#define MC_STACK_CAPACITY 64
// Child reference of an unused slot in a 4-wide node.
#define MC_WIDE_EMPTY 0x7FFFFFFF

namespace mc {

// Records the message for mc_last_error() and returns s.
mc_status set_error(mc_status s, const char* fmt, ...);
mc_status cuda_error(int err, const char* what, const char* file, int line);
mc_status status_from_device_flags(int flags);

void build_env_tables(const float* rgba, int W, int H, std::vector<float>& rowCdf, std::vector<float>& colCdf,
                      float& total);

// One entry of an environment map's alias table: keep texel i when a uniform
// draw is below threshold, else take texel alias.
struct EnvAliasEntry {
    float threshold;
    int32_t alias;
};
void build_env_alias(const std::vector<float>& colCdf, int W, int H, std::vector<EnvAliasEntry>& table);
// The device alias table of a map made by mc_env_create (EnvAliasEntry[width *
// height]), or null for a disabled map or one the library did not create.
const void* env_alias_table(const mc_env_map& env);

// Grow-only device buffer.
struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
};
mc_status devbuf_reserve(DevBuf& b, size_t bytes);
void devbuf_free(DevBuf& b);
// stream-ordered allocations from the device's pool (BVH build buffers)
mc_status pool_alloc(mc_context* ctx, void** p, size_t bytes);
void pool_free(mc_context* ctx, void* p);  // ordered after the work queued on ctx's stream
void pool_release(void* p);                // device current and its readers finished
void pool_trim(int device);                // hands the pool's unused memory back

// Copies `bytes` of host memory to the device; complete when the call returns.
// Large copies from pageable memory go through the context's pinned staging
// buffers, filled by several host threads while earlier pieces are in flight.
mc_status upload_host(mc_context* ctx, void* dst, const void* src, size_t bytes);

// Per-bounce counters of one sample: [d][0] extend-queue size of bounce d,
// [d][1] shadow-queue size of bounce d, [d][2] trace work counter,
// [d][3] medium pass-through count.
#define MC_COUNTERS_PER_DEPTH 4

struct WaveBuffers {
    int capacity = 0;
    // path state, SoA (PT:3138-3163 PathStateBuffers)
    float* ox = nullptr; float* oy = nullptr; float* oz = nullptr;
    float* dx = nullptr; float* dy = nullptr; float* dz = nullptr;
    float* time = nullptr;
    float* tr = nullptr; float* tg = nullptr; float* tb = nullptr;
    float* sr = nullptr; float* sg = nullptr; float* sb = nullptr;
    unsigned char* spec = nullptr;
    float* pdf = nullptr;
    uint32_t* draw = nullptr;          // Philox draw counter per path
    mc_packed_hit* hits = nullptr;     // PT:3165 HitResultBuffers
    int* queue[2] = {nullptr, nullptr};  // extend queues (ping-pong)
    // shadow-ray queue, SoA (PT:3170-3186 ShadowRayQueue)
    float* sox = nullptr; float* soy = nullptr; float* soz = nullptr;
    float* sdx = nullptr; float* sdy = nullptr; float* sdz = nullptr;
    float* smax = nullptr;
    float* scr = nullptr; float* scg = nullptr; float* scb = nullptr;
    int* spath = nullptr;
    DevBuf block;                      // one allocation backs all of the above
};

}  // namespace mc

struct mc_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    int sm_count = 0;
    int* d_error = nullptr;            // device error word
    int* d_wait_error = nullptr;       // error word of mc_stream_wait_value (read by mc_context_synchronize)
    long long wait_timeout_ns = 2000000000ll;  // bounded waits on external flags
    int* d_counters = nullptr;         // (MC_MAX_DEPTH_STATS+1) * MC_COUNTERS_PER_DEPTH ints
    long long* d_stats = nullptr;      // 2 * MC_MAX_DEPTH_STATS accumulated ray counts
    mc::DevBuf scratch[8];             // build / sort scratch
    mc::WaveBuffers wave;
    mc::DevBuf volume;                 // per shadow slot: medium crossings (scenes with density grids)
    void* rng_states = nullptr;        // curandState per pixel (XORWOW mode)
    int rng_pixels = 0;
    unsigned long long rng_seed = 0;
    bool rng_ready = false;
    // wave tables: device copy + a ring of pinned host tables (one per wave in flight)
    void* d_table = nullptr;
    void* h_tables = nullptr;
    void* table_events[4] = {nullptr, nullptr, nullptr, nullptr};
    int table_slot = 0;
    unsigned short* scene_of = nullptr;  // scene id per path (batched waves)
    int scene_of_capacity = 0;
    cudaStream_t own_stream = nullptr;   // capture stream when the context has none
    void* graph_exec = nullptr;          // cached per-wave CUDA graph
    unsigned long long graph_key[16] = {};  // every value the captured launches bake in
    void* staging = nullptr;             // pinned host staging for large pageable uploads
    size_t staging_bytes = 0;
    // launch configurations measured on this context's device (occupancy of a
    // kernel variant, its opt-in shared-memory size), filled on first use; a
    // context is used by one host thread at a time, so these need no lock
    int trace_blocks[144] = {};
    int trace_blocks_smem[144] = {};     // shared-memory bytes trace_blocks[k] was measured with
    int trace_smem_attr[144] = {};       // dynamic shared memory the variant has been opted in to
    int shade_blocks[3] = {};            // Philox, XORWOW, guided
    bool guide_attrs_set = false;        // the guide kernels' shared-memory opt-in is done
};

struct mc_bvh {
    mc_context* ctx = nullptr;
    int device = 0;
    int n = 0, ns = 0, nt = 0;
    int ni = 0;                        // internal binary nodes over all segments
    int nseg = 1;                      // scenes in this build (a batch build has several)
    std::vector<int> seg_prim_off;     // first leaf (primitive record) index of each scene
    std::vector<int> bin_roots;        // binary root node of each scene
    std::vector<int> wide_roots;       // 4-wide root node of each scene
    std::vector<mc_aabb> seg_bounds;   // root box of each scene
    int layout = MC_BVH_LAYOUT_BINARY;
    int builder = MC_BVH_BUILDER_LBVH;  // the binary tree the wide layout collapses
    int depth = -1;
    void* nodes = nullptr;             // traversal nodes (float4 records)
    long long node_count = 0;
    long long node_bytes = 0;
    void* prims = nullptr;             // leaf-ordered primitive records, 48 B each
    void* wide_nodes = nullptr;        // 4-wide nodes, 128 B each (layout MC_BVH_LAYOUT_WIDE4)
    long long wide_count = 0;
    int wide_levels = -1;              // levels of the greedy 4-wide tree (a ray's stack holds <= 3 per level), -1 unknown
    void* wide_prims = nullptr;        // primitive records in reference visit (rank) order
    // reference representation (optional)
    uint32_t* codes = nullptr;
    int32_t* ids = nullptr;
    int32_t* types = nullptr;
    mc_bvh_node* ref_internal = nullptr;
    mc_bvh_node* ref_leaves = nullptr;
    int32_t* parents = nullptr;        // internal parents (n-1) then leaf parents (n), encoded (p<<1)|side
    mc_aabb bounds;
};

struct mc_guide {
    mc_context* ctx = nullptr;
    mc_guide_config cfg;
    float* master = nullptr;           // FP32 parameters
    float* adam_m = nullptr;
    float* adam_v = nullptr;
    void* blob = nullptr;              // BF16 weights (forward and transposed copies)
    float* partials = nullptr;         // per-CTA gradient partials [sm_count][PARAM_COUNT]
    float* scale = nullptr;            // device: weight normalization of the current step
    double* loss = nullptr;            // device: loss accumulator
    float* batch = nullptr;            // training records of guided renders
    int batch_records = 0;             // records the batch buffer holds
    int* batch_count = nullptr;
    int* rec_tiles = nullptr;          // per-tile record counts, then first batch slots, of a wave
    int rec_tile_capacity = 0;
    float* records = nullptr;          // per-path primary-vertex records of guided renders
    int record_capacity = 0;
    float* mixtures = nullptr;         // per-path mixtures of the current bounce
    int mixture_capacity = 0;
    float* nee0 = nullptr;             // per-path NEE of the primary vertex (kept out of the records' weights)
    int steps = 0;
};

namespace mc {

struct RenderTiming {
    float ms = 0.f;
    float trace_ms = 0.f;
    float shade_ms = 0.f, infer_ms = 0.f, train_ms = 0.f;
    int trace_launches = 0;
    int kernel_launches = 0;
};

// One image of a wave sequence: its scene arrays, parameters, accumulation
// buffer and BVH root; bvh, when set, is this item's own BVH (the server's
// per-scene trees) instead of the segment of the shared one.
struct WaveItem {
    const mc_scene_view* view;
    const mc_render_params* p;
    float* accum;
    int root;
    int segment;
    const mc_bvh* bvh = nullptr;
    // Samples of this item traced together in one wave (pixel-major: the
    // samples of a pixel are neighbouring paths). Counter-based RNG only.
    int spw = 1;
};

// Renders the items' samples in shared waves (mc_render.cu).
mc_status run_waves(mc_context* ctx, const mc_bvh* bvh, const WaveItem* items, int n, bool useGraph, bool timed,
                    RenderTiming* tm, mc_guide* guide = nullptr, bool train = false);
// run_waves with the error word and ray statistics reset before and read after.
mc_status render_items(mc_context* ctx, const mc_bvh* bvh, const WaveItem* items, int n, bool useGraph,
                       mc_render_stats* stats, mc_guide* guide = nullptr, bool train = false);
mc_status check_params(const mc_render_params* p, const mc_scene_view* v);

mc_status bvh_depth(mc_bvh* bvh);
mc_status context_counters(mc_context* ctx);
// Guide kernels driven by device-side counts (guided renders).
// Inputs of a queued path: its hit point and, per the guide's direction_input,
// the face normal of the hit primitive (hot, spheres, time) or the ray direction.
// stride > 1: only every stride-th queue slot is queried (the first sample of
// each pixel of a pixel-major wave at bounce 0; its samples share the mixture).
mc_status guide_infer_paths(mc_guide* g, cudaStream_t s, const int* queue, const int* count, int capacity,
                            const float* ox, const float* oy, const float* oz, const float* dx, const float* dy,
                            const float* dz, const float* time, const mc_packed_hit* hits, const mc_triangle_hot* hot,
                            const mc_sphere* spheres, float* mixtures, int stride = 1);
// `steps` Adam steps, each on the next min(stepRecords, cfg.batch_capacity)
// of the records (stepRecords <= 0: cfg.batch_capacity).
mc_status guide_train_device(mc_guide* g, cudaStream_t s, const float* records, const int* count, int capacity, int steps,
                             int stepRecords);
// Grows the training batch buffer to hold `records` records.
mc_status guide_reserve_batch(mc_guide* g, int records);
mc_status guide_reserve_tiles(mc_guide* g, int tiles);
// Samples per pixel in one wave of a single-image render of these params.
int wave_samples(const mc_render_params* params);
mc_status guide_reserve_paths(mc_guide* g, int paths);
}
