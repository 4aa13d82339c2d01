// mc_server.cu - a render server over the wavefront path: resident scenes and
// BVHs, admission by an HBM budget, and shared waves for all active requests.
//
// Each step renders samples_per_step samples of every active request. Plain
// requests of every scene go into the same waves: the wave table holds one
// entry per request (its own BVH, scene arrays, camera, image and sample
// number), so one persistent trace launch and one shade launch per bounce
// serve all of them. Guided requests render with their scene's guide, which
// keeps training online across requests of that scene.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <vector>

#include "mc_internal.h"

namespace {

// Wave-buffer bytes per path (path state, queues, shadow queue, hits, scene id)
// and the guide's per-path buffers (mixture, record, primary NEE).
constexpr long long kWaveBytesPerPath = 29 * 4 + 1 + 16 + 2;
constexpr long long kGuideBytesPerPath = (40 + 12 + 3) * 4;
// scenes with density grids: per shadow slot the medium crossings (36 B) and
// a place in the list of rays that crossed a grid (4 B)
constexpr long long kGridBytesPerPath = 40;

struct ServerScene {
    mc_scene_view view;
    mc_bvh* bvh = nullptr;
    mc_guide* guide = nullptr;
    long long bytes = 0;
};

struct ServerRequest {
    long long id = 0;
    long long scene = 0;
    mc_render_params params;
    bool guided = false;
    int state = MC_REQ_PENDING;
    int done = 0;
    float* accum = nullptr;
    long long bytes = 0;
    double submit_s = 0, admit_s = 0, done_s = 0;
};

long long bvh_bytes(const mc_bvh* b) {
    long long n = b->n;
    long long s = b->node_bytes + n * 48 + b->wide_count * 128 + n * 48 + 3 * n * 4 + (2 * n) * 4;
    if (b->ref_internal) s += (2 * n) * (long long)sizeof(mc_bvh_node);
    return s;
}

}  // namespace

struct mc_server {
    mc_context* ctx = nullptr;
    int device = 0;
    mc_server_config cfg;
    std::chrono::steady_clock::time_point t0;
    std::vector<ServerScene> scenes;
    std::map<long long, ServerRequest> requests;
    std::deque<long long> pending;
    std::vector<long long> active;
    long long next_id = 1;
    long long used = 0;
    long long scene_bytes = 0;
    long long steps = 0, waves = 0, rays = 0;
    int done = 0;

    double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
};

namespace {

// A plain request traces its step's samples in one wave (one path per pixel
// and sample); a guided one a sample per wave.
long long request_bytes(const mc_render_params& p, bool guided, int sps, bool grid) {
    long long px = (long long)p.width * p.height;
    long long spw = guided ? 1 : std::max(1, std::min(sps, p.spp));
    return px * 12 + px * spw * (kWaveBytesPerPath + (grid ? kGridBytesPerPath : 0)) +
           (guided ? px * kGuideBytesPerPath : 0);
}

mc_status admit(mc_server* s) {
    const double t = s->now();
    while (!s->pending.empty() && (int)s->active.size() < s->cfg.max_active) {
        ServerRequest& r = s->requests[s->pending.front()];
        if (s->used + r.bytes > s->cfg.hbm_budget_bytes) break;  // arrival order: the head waits for room
        size_t accBytes = (size_t)r.params.width * r.params.height * 3 * sizeof(float);
        // from the device's stream-ordered pool: a driver allocation per
        // request costs up to hundreds of milliseconds at random
        if (mc::pool_alloc(s->ctx, (void**)&r.accum, accBytes) != MC_OK)
            return mc::set_error(MC_ERR_OOM, "mc_server_step: accumulation buffer allocation failed");
        cudaMemsetAsync(r.accum, 0, accBytes, s->ctx->stream);
        s->used += r.bytes;
        r.state = MC_REQ_ACTIVE;
        r.admit_s = t;
        s->active.push_back(r.id);
        s->pending.pop_front();
    }
    return MC_OK;
}

}  // namespace

extern "C" {

mc_status mc_server_create(mc_context* ctx, const mc_server_config* config, mc_server** out) {
    if (!ctx || !out) return mc::set_error(MC_ERR_INVALID, "mc_server_create: null argument");
    mc_server* s = new mc_server();
    s->ctx = ctx;
    s->device = ctx->device;
    if (config) s->cfg = *config;
    else std::memset(&s->cfg, 0, sizeof(s->cfg));
    if (s->cfg.hbm_budget_bytes <= 0) s->cfg.hbm_budget_bytes = 150ll * 1000 * 1000 * 1000;
    if (s->cfg.max_active <= 0) s->cfg.max_active = 128;
    if (s->cfg.max_active > 128) s->cfg.max_active = 128;
    if (s->cfg.samples_per_step <= 0) s->cfg.samples_per_step = 16;
    if (s->cfg.wave_paths <= 0) s->cfg.wave_paths = 4194304;
    s->t0 = std::chrono::steady_clock::now();
    *out = s;
    return MC_OK;
}

// Does not touch the server's context (which may be gone already): the
// accumulation buffers go back to the pool once the device's work is done.
mc_status mc_server_destroy(mc_server* s) {
    if (!s) return MC_OK;
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != s->device) cudaSetDevice(s->device);
    cudaDeviceSynchronize();
    for (auto& kv : s->requests) mc::pool_release(kv.second.accum);
    if (prev >= 0 && prev != s->device) cudaSetDevice(prev);
    for (auto& sc : s->scenes) {
        mc_bvh_free(sc.bvh);
        mc_guide_destroy(sc.guide);
    }
    delete s;
    return MC_OK;
}

mc_status mc_server_add_scene(mc_server* s, const mc_scene_view* scene, int64_t* scene_id) {
    if (!s || !scene || !scene_id) return mc::set_error(MC_ERR_INVALID, "mc_server_add_scene: null argument");
    mc_bvh_build_opts opts;
    std::memset(&opts, 0, sizeof(opts));
    opts.layout = MC_BVH_LAYOUT_WIDE4;
    ServerScene sc;
    sc.view = *scene;
    mc_status st = mc_bvh_build(s->ctx, scene, &opts, &sc.bvh);
    if (st != MC_OK) return st;
    sc.bytes = bvh_bytes(sc.bvh);
    if (s->used + sc.bytes > s->cfg.hbm_budget_bytes) {
        mc_bvh_free(sc.bvh);
        return mc::set_error(MC_ERR_BUDGET, "mc_server_add_scene: the scene's BVH (%lld bytes) does not fit the budget",
                             sc.bytes);
    }
    s->used += sc.bytes;
    s->scene_bytes += sc.bytes;
    s->scenes.push_back(sc);
    *scene_id = (int64_t)s->scenes.size() - 1;
    return MC_OK;
}

mc_status mc_server_submit(mc_server* s, const mc_server_request* req, int64_t* request_id) {
    if (!s || !req || !request_id) return mc::set_error(MC_ERR_INVALID, "mc_server_submit: null argument");
    if (req->scene_id < 0 || req->scene_id >= (int64_t)s->scenes.size())
        return mc::set_error(MC_ERR_NOT_FOUND, "mc_server_submit: unknown scene %lld", (long long)req->scene_id);
    const ServerScene& sc = s->scenes[(size_t)req->scene_id];
    mc_status st = mc::check_params(&req->params, &sc.view);
    if (st != MC_OK) return st;
    if (req->params.rng != MC_RNG_PHILOX) return mc::set_error(MC_ERR_INVALID, "mc_server_submit: requests use the counter-based RNG");
    if (req->params.spp < 1) return mc::set_error(MC_ERR_INVALID, "mc_server_submit: spp must be >= 1");
    ServerRequest r;
    r.id = s->next_id++;
    r.scene = req->scene_id;
    r.params = req->params;
    r.guided = req->guided != 0;
    r.bytes = request_bytes(r.params, r.guided, s->cfg.samples_per_step, (sc.view.has_medium & MC_MEDIUM_GRID) != 0);
    if (r.bytes + s->scene_bytes > s->cfg.hbm_budget_bytes)
        return mc::set_error(MC_ERR_BUDGET, "mc_server_submit: the request needs %lld bytes, more than the budget leaves",
                             r.bytes);
    r.submit_s = s->now();
    s->requests[r.id] = r;
    s->pending.push_back(r.id);
    *request_id = r.id;
    return MC_OK;
}

mc_status mc_server_step(mc_server* s, int32_t* active_out) {
    if (!s) return mc::set_error(MC_ERR_INVALID, "mc_server_step: null server");
    mc_status st = admit(s);
    if (st != MC_OK) return st;
    s->steps++;
    const int sps = s->cfg.samples_per_step;
    // schedule: the oldest active request (no starvation), then least remaining
    // work first while the step's paths stay within wave_paths
    std::vector<long long> order(s->active.begin(), s->active.end());
    if (order.size() > 1) {
        std::stable_sort(order.begin() + 1, order.end(), [&](long long a, long long b) {
            const ServerRequest& ra = s->requests[a];
            const ServerRequest& rb = s->requests[b];
            long long wa = (long long)ra.params.width * ra.params.height * (ra.params.spp - ra.done);
            long long wb = (long long)rb.params.width * rb.params.height * (rb.params.spp - rb.done);
            return wa < wb;
        });
    }
    std::vector<long long> chosen;
    long long paths = 0;
    for (long long id : order) {
        const ServerRequest& r = s->requests[id];
        long long px = (long long)r.params.width * r.params.height;
        if (!chosen.empty() && paths + px > s->cfg.wave_paths) continue;
        chosen.push_back(id);
        paths += px;
    }
    // plain requests: every scene's in one shared wave (the trace looks up each
    // ray's scene), or with MC_SERVER_SCENE_WAVES one wave per scene (single-scene
    // trace launches, which can take the 128-thread block shape with the stack
    // that scene's tree needs)
    std::map<long long, std::vector<long long>> plainGroups;
    const bool sceneWaves = (s->cfg.flags & MC_SERVER_SCENE_WAVES) != 0;
    for (long long id : chosen) {
        const ServerRequest& r = s->requests[id];
        if (r.guided) continue;
        plainGroups[sceneWaves ? r.scene : -1].push_back(id);
    }
    for (auto& grp : plainGroups) {
        const std::vector<long long>& ids = grp.second;
        long long oneScene = s->requests[ids[0]].scene;
        for (long long id : ids)
            if (s->requests[id].scene != oneScene) oneScene = -1;
        int stackNeed = 0;
        if (oneScene >= 0) {
            const int lv = s->scenes[(size_t)oneScene].bvh->wide_levels;
            if (lv > 0) stackNeed = ((3 * lv + 7) / 8) * 8;
        }
        std::vector<mc_render_params> params;
        std::vector<mc::WaveItem> items;
        params.reserve(ids.size());
        for (long long id : ids) {
            ServerRequest& r = s->requests[id];
            mc_render_params p = r.params;
            p.first_sample = r.params.first_sample + r.done;
            p.spp = std::min(sps, r.params.spp - r.done);
            p.use_graph = 0;
            p.instrument = 0;
            // launch shape (the image does not depend on it): the refill threshold
            // and block shape the autotuner picks for large scenes, unless the
            // request set its own
            if (p.refill_threshold <= 0) p.refill_threshold = 16;
            if (p.trace_threads == 0 && stackNeed > 0 && stackNeed <= 56 && p.stack_entries == 0 &&
                p.intersector == MC_ISECT_REFERENCE) {
                p.trace_threads = 128;
                p.stack_entries = stackNeed;
            }
            params.push_back(p);
        }
        for (size_t i = 0; i < ids.size(); i++) {
            ServerRequest& r = s->requests[ids[i]];
            const ServerScene& sc = s->scenes[(size_t)r.scene];
            mc::WaveItem it{&sc.view, &params[i], r.accum, sc.bvh->wide_roots[0], 0};
            it.bvh = sc.bvh;
            it.spw = params[i].spp;  // the step's samples in one wave, pixel-major
            items.push_back(it);
        }
        mc_render_stats rs;
        st = mc::render_items(s->ctx, items[0].bvh, items.data(), (int)items.size(), false, &rs);
        if (st != MC_OK) return st;
        s->rays += rs.extend_rays + rs.shadow_rays;
        s->waves += 1;  // each request's step samples share the one wave
        for (size_t i = 0; i < ids.size(); i++) s->requests[ids[i]].done += params[i].spp;
    }
    // guided requests: the ones of each scene share waves and the scene's
    // guide, which trains on all of their primary vertices
    std::map<long long, std::vector<long long>> guidedByScene;
    for (long long id : chosen)
        if (s->requests[id].guided) guidedByScene[s->requests[id].scene].push_back(id);
    for (auto& kv : guidedByScene) {
        ServerScene& sc = s->scenes[(size_t)kv.first];
        if (!sc.guide) {
            mc_guide_config gc;
            std::memset(&gc, 0, sizeof(gc));
            gc.bounds = sc.bvh->bounds;
            gc.seed = (uint64_t)kv.first + 1;
            // a scene's guide lives as long as the scene and keeps training on
            // every guided request; the default guide (anchored lobes, first
            // bounce guided and trained) is the one that reached plain's error
            // fastest once trained (about 0.8x plain's time on the aperture room)
            if ((st = mc_guide_create(s->ctx, &gc, &sc.guide)) != MC_OK) return st;
        }
        std::vector<mc_render_params> gp;
        std::vector<mc::WaveItem> gi;
        gp.reserve(kv.second.size());
        int paths = 0, w = 0;
        for (long long id : kv.second) {
            ServerRequest& r = s->requests[id];
            mc_render_params p = r.params;
            p.first_sample = r.params.first_sample + r.done;
            p.spp = std::min(sps, r.params.spp - r.done);
            p.use_graph = 0;
            p.instrument = 0;
            gp.push_back(p);
            paths += p.width * p.height;
            w = std::max(w, p.spp);
        }
        for (size_t i = 0; i < kv.second.size(); i++) {
            ServerRequest& r = s->requests[kv.second[i]];
            mc::WaveItem it{&sc.view, &gp[i], r.accum, sc.bvh->wide_roots[0], 0};
            it.bvh = sc.bvh;
            gi.push_back(it);
        }
        if ((st = mc::guide_reserve_paths(sc.guide, paths)) != MC_OK) return st;
        mc_render_stats rs;
        st = mc::render_items(s->ctx, sc.bvh, gi.data(), (int)gi.size(), false, &rs, sc.guide, true);
        if (st != MC_OK) return st;
        s->rays += rs.extend_rays + rs.shadow_rays;
        s->waves += w;
        for (size_t i = 0; i < kv.second.size(); i++) s->requests[kv.second[i]].done += gp[i].spp;
    }
    // retire finished requests (their buffers stay until released)
    const double t = s->now();
    std::vector<long long> still;
    for (long long id : s->active) {
        ServerRequest& r = s->requests[id];
        if (r.done >= r.params.spp) {
            r.state = MC_REQ_DONE;
            r.done_s = t;
            s->done++;
        } else {
            still.push_back(id);
        }
    }
    s->active.swap(still);
    if (active_out) *active_out = (int32_t)s->active.size();
    return MC_OK;
}

mc_status mc_server_get_result(mc_server* s, int64_t request_id, mc_server_result* out) {
    if (!s || !out) return mc::set_error(MC_ERR_INVALID, "mc_server_get_result: null argument");
    auto it = s->requests.find(request_id);
    if (it == s->requests.end()) return mc::set_error(MC_ERR_NOT_FOUND, "mc_server_get_result: unknown request %lld", (long long)request_id);
    const ServerRequest& r = it->second;
    std::memset(out, 0, sizeof(*out));
    out->request_id = r.id;
    out->state = r.state;
    out->spp_done = r.done;
    out->submit_s = r.submit_s;
    out->admit_s = r.admit_s;
    out->done_s = r.done_s;
    out->bytes = r.bytes;
    out->d_accum = r.accum;
    return MC_OK;
}

mc_status mc_server_read(mc_server* s, int64_t request_id, float* host_rgb) {
    if (!s || !host_rgb) return mc::set_error(MC_ERR_INVALID, "mc_server_read: null argument");
    auto it = s->requests.find(request_id);
    if (it == s->requests.end()) return mc::set_error(MC_ERR_NOT_FOUND, "mc_server_read: unknown request %lld", (long long)request_id);
    const ServerRequest& r = it->second;
    if (r.state == MC_REQ_CANCELLED) return mc::set_error(MC_ERR_CANCELLED, "mc_server_read: request %lld was cancelled", (long long)request_id);
    if (!r.accum) return mc::set_error(MC_ERR_INVALID, "mc_server_read: request %lld holds no image", (long long)request_id);
    const size_t bytes = (size_t)r.params.width * r.params.height * 3 * sizeof(float);
    cudaError_t e = cudaMemcpyAsync(host_rgb, r.accum, bytes, cudaMemcpyDeviceToHost, s->ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->ctx->stream);
    if (e != cudaSuccess) return mc::cuda_error((int)e, "mc_server_read", __FILE__, __LINE__);
    return MC_OK;
}

mc_status mc_server_encode(mc_server* s, int64_t request_id, const mc_image_options* opts, void* out, int64_t* bytes,
                           float* chosen_exposure) {
    if (!s || !opts || !bytes) return mc::set_error(MC_ERR_INVALID, "mc_server_encode: null argument");
    if (opts->device_output) return mc::set_error(MC_ERR_INVALID, "mc_server_encode: the response goes to host memory");
    auto it = s->requests.find(request_id);
    if (it == s->requests.end()) return mc::set_error(MC_ERR_NOT_FOUND, "mc_server_encode: unknown request %lld", (long long)request_id);
    const ServerRequest& r = it->second;
    if (r.state == MC_REQ_CANCELLED) return mc::set_error(MC_ERR_CANCELLED, "mc_server_encode: request %lld was cancelled", (long long)request_id);
    if (!r.accum) return mc::set_error(MC_ERR_INVALID, "mc_server_encode: request %lld holds no image", (long long)request_id);
    if (r.done <= 0) return mc::set_error(MC_ERR_INVALID, "mc_server_encode: request %lld has no samples yet", (long long)request_id);
    return mc_image_encode(s->ctx, r.accum, r.params.width, r.params.height, r.done, opts, out, bytes, chosen_exposure);
}

mc_status mc_server_release(mc_server* s, int64_t request_id) {
    if (!s) return mc::set_error(MC_ERR_INVALID, "mc_server_release: null server");
    auto it = s->requests.find(request_id);
    if (it == s->requests.end()) return mc::set_error(MC_ERR_NOT_FOUND, "mc_server_release: unknown request %lld", (long long)request_id);
    ServerRequest& r = it->second;
    if (r.state == MC_REQ_CANCELLED) return MC_OK;  // its memory went back when it was cancelled
    if (r.state != MC_REQ_DONE) return mc::set_error(MC_ERR_INVALID, "mc_server_release: request %lld is not done", (long long)request_id);
    mc::pool_free(s->ctx, r.accum);  // after the work queued on the server's stream
    r.accum = nullptr;
    r.state = MC_REQ_RELEASED;
    s->used -= r.bytes;
    return MC_OK;
}

mc_status mc_server_cancel(mc_server* s, int64_t request_id) {
    if (!s) return mc::set_error(MC_ERR_INVALID, "mc_server_cancel: null server");
    auto it = s->requests.find(request_id);
    if (it == s->requests.end()) return mc::set_error(MC_ERR_NOT_FOUND, "mc_server_cancel: unknown request %lld", (long long)request_id);
    ServerRequest& r = it->second;
    if (r.state == MC_REQ_PENDING) {
        s->pending.erase(std::remove(s->pending.begin(), s->pending.end(), r.id), s->pending.end());
    } else if (r.state == MC_REQ_ACTIVE) {
        s->active.erase(std::remove(s->active.begin(), s->active.end(), r.id), s->active.end());
        // steps are synchronous, so no launch of this request is in flight;
        // the stream-ordered free would follow one all the same
        mc::pool_free(s->ctx, r.accum);
        r.accum = nullptr;
        s->used -= r.bytes;
    } else {
        return mc::set_error(r.state == MC_REQ_CANCELLED ? MC_ERR_CANCELLED : MC_ERR_INVALID,
                             "mc_server_cancel: request %lld is %s", (long long)request_id,
                             r.state == MC_REQ_CANCELLED ? "already cancelled" : "done");
    }
    r.state = MC_REQ_CANCELLED;
    r.done_s = s->now();
    return MC_OK;
}

mc_status mc_server_get_stats(const mc_server* s, mc_server_stats* out) {
    if (!s || !out) return mc::set_error(MC_ERR_INVALID, "mc_server_get_stats: null argument");
    std::memset(out, 0, sizeof(*out));
    out->budget_bytes = s->cfg.hbm_budget_bytes;
    out->used_bytes = s->used;
    out->scene_bytes = s->scene_bytes;
    out->scenes = (int32_t)s->scenes.size();
    out->pending = (int32_t)s->pending.size();
    out->active = (int32_t)s->active.size();
    out->done = s->done;
    out->steps = s->steps;
    out->waves = s->waves;
    out->rays = s->rays;
    return MC_OK;
}

double mc_server_now(const mc_server* s) { return s ? s->now() : 0.0; }

}  // extern "C"
