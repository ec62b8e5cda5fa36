// serve.cuh — render server with continuous batching (part of the render.cu
// translation unit: it drives the same kernels).
//
// A worker thread owns the context's stream.  Each iteration it
//   1. admits queued requests while their framebuffer and path-state
//      ranges fit the pooled device memory (the HBM budget set at creation)
//      and a view slot is free (a request that does not fit is passed over
//      for a bounded time); each admitted request writes its view into the
//      device view table; primary passes (with each new path's first
//      shading step) start up to a per-step path budget of tiles and append
//      the paths to the shared live-path queue;
//   2. runs one shade pass and one trace pass over every live path — paths of
//      all admitted requests at whatever bounce they are — so a request that
//      arrives while others are on the GPU joins at the next pass;
//   3. reads the per-slot counts of paths not yet deposited; a request whose
//      count reached zero is resolved (AvgPass + tonemap over its pixels) on
//      the render stream, and its images are copied to the caller's host
//      buffers on the server's copy stream while the next steps render; its
//      pool ranges and view slot are released once that copy has ended.
// Scenes and their radiance caches stay resident in the context.  The
// per-frame cache decay of ve_render does not apply: requests accumulate into
// the persistent per-scene caches.
#pragma once
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <thread>
#include <unordered_map>

namespace ve {

// First-fit allocator of contiguous ranges in [0, capacity).
class RangePool {
public:
    explicit RangePool(uint64_t cap = 0) { reset(cap); }
    void reset(uint64_t cap) {
        free_.clear();
        if (cap) free_[0] = cap;
        cap_ = cap;
        used_ = 0;
    }
    bool alloc(uint64_t n, uint64_t* off) {
        if (n == 0) n = 1;
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= n) {
                *off = it->first;
                const uint64_t rest = it->second - n, start = it->first + n;
                free_.erase(it);
                if (rest) free_[start] = rest;
                used_ += n;
                return true;
            }
        }
        return false;
    }
    void release(uint64_t off, uint64_t n) {
        if (n == 0) n = 1;
        used_ -= n;
        auto it = free_.emplace(off, n).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
    uint64_t used() const { return used_; }
    uint64_t capacity() const { return cap_; }

private:
    std::map<uint64_t, uint64_t> free_;
    uint64_t cap_ = 0, used_ = 0;
};

struct ServeRequest {
    uint64_t id = 0;
    ve_view view{};
    uint32_t* out_vid = nullptr;
    float* out_rgb = nullptr;
    int state = 0;  // 0 queued, 1 on the GPU, 2 resolving, 3 done, 4 failed
    uint32_t slot = 0;
    uint64_t pix_off = 0, path_off = 0, pixels = 0, paths = 0;
    uint32_t tiles = 0;
    uint32_t tiles_started = 0;  // tiles whose primary pass has been launched
    double t_submit = 0, t_admit = 0, t_done = 0;
    cudaEvent_t done_ev = nullptr;
    ve_server* owner = nullptr;
};

inline double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace ve

struct ve_server {
    ve_ctx* c = nullptr;
    ve_server_config cfg{};
    std::thread worker;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    bool stop = false;
    int error = VE_OK;
    std::string error_msg;
    uint64_t next_id = 1;
    std::deque<ve::ServeRequest*> queue;
    std::vector<ve::ServeRequest*> active;
    std::unordered_map<uint64_t, ve::ServeRequest*> all;
    std::vector<uint32_t> free_slots;
    ve::RangePool pix_pool, path_pool;
    uint32_t* d_remaining = nullptr;
    uint32_t* h_remaining = nullptr;  // pinned
    unsigned long long* h_stats = nullptr;  // pinned copy of the context's per-kind ray counters
    ve::DevView* h_view = nullptr;    // pinned staging, one per slot
    cudaStream_t copy_st = nullptr;   // output copies of finished requests
    cudaEvent_t resolve_ev = nullptr; // the resolves the next copies wait for
    uint64_t step = 0;
    // stats
    uint64_t completed = 0, steps_run = 0, max_inflight = 0, admitted = 0, rays = 0;
};

namespace ve {

static void serve_fail(ve_server* s, int code, const std::string& msg) {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->error == VE_OK) {
        s->error = code;
        s->error_msg = msg;
    }
    s->stop = true;
    s->cv_done.notify_all();
}

// Host function on the copy stream after a finished request's output
// copies: the request is done, its pool ranges and view slot return to the
// free lists, and waiters (and an idle serve loop) are woken.  Runs on a
// CUDA-internal thread: no CUDA calls, only the server's lock.
static void CUDART_CB serve_copied(void* arg) {
    ServeRequest* r = static_cast<ServeRequest*>(arg);
    ve_server* s = r->owner;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        r->state = 3;
        r->t_done = now_s();
        s->pix_pool.release(r->pix_off, r->pixels);
        s->path_pool.release(r->path_off, r->paths);
        s->free_slots.push_back(r->slot);
        s->active.erase(std::find(s->active.begin(), s->active.end(), r));
        s->completed++;
    }
    s->cv_done.notify_all();
    s->cv_work.notify_all();
}

static FrameArgs serve_args(ve_server* s) {
    ve_ctx* c = s->c;
    FrameArgs a{};
    a.views = c->d_views.p;
    a.n_views = s->cfg.max_requests;
    a.scenes = c->d_scenes.p;
    a.mats = c->d_mats.p;
    a.p_ray_o = c->p_ray_o.p; a.p_ray_d = c->p_ray_d.p; a.p_tp = c->p_tp.p;
    a.p_direct = c->p_direct.p; a.p_indirect = c->p_indirect.p; a.p_pend = c->p_pend.p;
    a.p_hit = c->p_hit.p; a.p_meta = c->p_meta.p;
    a.live[0] = c->live0.p; a.live[1] = c->live1.p; a.rayq = c->rayq.p;
    a.rayq_sh = c->rayq.p + s->cfg.path_capacity;
    a.counters = c->counters.p; a.stats = c->stats.p;
    a.gbuf = c->gbuf.p; a.out_vid = c->out_vid.p; a.out_node = c->out_node.p;
    a.out_rgb = c->out_rgb.p; a.out_mapped = c->out_mapped.p;
    a.path_rgb = nullptr;
    a.refill = c->launch.refill_threshold;
    a.view_offset = 0;
    a.remaining = s->d_remaining;
    return a;
}

static void serve_loop(ve_server* s) {
    ve_ctx* c = s->c;
    cudaSetDevice(c->device);
    cudaStream_t st = c->stream;
    constexpr uint32_t kRing = 16;  // counter slots per pass index (even: keeps the live ping-pong parity)
    for (;;) {
        std::vector<ServeRequest*> admit, run;  // run: requests with paths to trace or tiles to start
        {
            std::unique_lock<std::mutex> lk(s->mu);
            // idle (or only output copies outstanding): wait for a request
            // or for a copy to end
            auto busy = [&] {
                for (ServeRequest* r : s->active)
                    if (r->state == 1) return true;
                return false;
            };
            if (s->queue.empty() && !busy()) {
                if (s->stop && s->active.empty()) break;
                s->cv_work.wait(lk, [&] { return (s->stop && s->active.empty()) || !s->queue.empty(); });
                if (s->stop && s->queue.empty() && s->active.empty()) break;
            }
            // 1. admission in arrival order while a slot is free; a request
            // that does not fit the pools is passed over unless it has waited
            // longer than the bypass bound (strict FIFO: never)
            const bool fifo = (s->cfg.flags & VE_SERVER_FIFO) != 0u;
            const double bypass_s = 1e-3 * double(s->cfg.max_bypass_ms ? s->cfg.max_bypass_ms : 50u);
            const double t_now = now_s();
            for (auto it = s->queue.begin(); it != s->queue.end() && !s->free_slots.empty();) {
                ServeRequest* r = *it;
                uint64_t po = 0, qo = 0;
                bool fits = s->pix_pool.alloc(r->pixels, &po);
                if (fits && !s->path_pool.alloc(r->paths, &qo)) {
                    s->pix_pool.release(po, r->pixels);
                    fits = false;
                }
                if (!fits) {
                    if (fifo || t_now - r->t_submit > bypass_s) break;
                    ++it;
                    continue;
                }
                it = s->queue.erase(it);
                r->pix_off = po;
                r->path_off = qo;
                r->slot = s->free_slots.back();
                s->free_slots.pop_back();
                r->state = 1;
                r->t_admit = now_s();
                s->active.push_back(r);
                admit.push_back(r);
                s->admitted++;
            }
            s->max_inflight = std::max<uint64_t>(s->max_inflight, s->active.size());
            for (ServeRequest* r : s->active)
                if (r->state == 1) run.push_back(r);
        }
        if (run.empty()) {
            // queued requests that do not fit wait for copies to free pool space
            std::unique_lock<std::mutex> lk(s->mu);
            const uint64_t done0 = s->completed;
            const size_t q0 = s->queue.size();
            s->cv_work.wait_for(lk, std::chrono::milliseconds(5),
                                [&] { return s->stop || s->completed != done0 || s->queue.size() != q0; });
            continue;
        }
        const uint32_t ps = uint32_t(s->step % kRing);
        // counters produced by this step's passes; the live count of slot
        // `ps` holds the previous shade's survivors (plus this step's new
        // primaries) and is kept.  Shade writes its survivor count at ps + 1.
        cudaMemsetAsync(c->counters.p + CNT_LIVE + ps + 1, 0, 4, st);
        cudaMemsetAsync(c->counters.p + CNT_RAY + ps, 0, 4, st);
        cudaMemsetAsync(c->counters.p + CNT_RAYSH + ps, 0, 4, st);
        cudaMemsetAsync(c->counters.p + CNT_CURSOR + ps, 0, 4, st);
        FrameArgs a = serve_args(s);
        for (ServeRequest* r : admit) {
            DevView& d = s->h_view[r->slot];
            const ve_view& v = r->view;
            const ve_frame_config& f = v.frame;
            std::memset(&d, 0, sizeof(d));
            std::memcpy(d.cam, v.camera, sizeof(d.cam));
            d.scene = uint32_t(v.scene_id);
            d.W = f.width; d.H = f.height; d.spp = f.spp;
            d.bounces = f.bounces; d.cc_primary = f.primary_controlchecks; d.cc_bounce = f.bounce_controlchecks;
            d.recon_radius = f.reconstruction_radius; d.render_type = f.render_type; d.frame_index = f.frame_index;
            // served requests render the plain method
            d.flags = f.flags & ~(VE_FRAME_PATH_RGB | VE_FRAME_SCHEDULED | VE_FRAME_EMISSIVE | VE_FRAME_LBUFFER |
                                  VE_FRAME_SPLIT | VE_FRAME_LEARNED | VE_FRAME_TRAIN | VE_FRAME_TERMINATE_HASH);
            set_rows(d, f, false);
            d.tiles_x = (f.width + 15) / 16;
            for (int k = 0; k < 3; k++) { d.sun[k] = f.sun_dir[k]; d.sky[k] = f.sky[k]; }
            d.sun_intensity = f.sun_intensity;
            d.decay = 1.0f;
            d.variance_norm = f.variance_norm;
            d.pix_base = uint32_t(r->pix_off);
            d.tile_base = 0;
            d.path_base = r->path_off;
            cudaMemcpyAsync(c->d_views.p + r->slot, &d, sizeof(DevView), cudaMemcpyHostToDevice, st);
            cudaMemsetAsync(s->d_remaining + r->slot, 0, 4, st);
        }
        // primary passes: requests in admission order start their next tiles
        // until the step's path budget is spent (FIFO: whole requests)
        {
            const bool fifo = (s->cfg.flags & VE_SERVER_FIFO) != 0u;
            uint64_t budget = s->cfg.step_path_budget ? s->cfg.step_path_budget : (1ull << 23);
            for (ServeRequest* r : run) {
                if (r->tiles_started >= r->tiles) continue;
                if (!fifo && budget == 0) break;
                const uint64_t per_tile = 256ull * r->view.frame.spp;
                const uint32_t left = r->tiles - r->tiles_started;
                uint32_t n = left;
                if (!fifo) n = uint32_t(std::min<uint64_t>(left, std::max<uint64_t>(1, budget / per_tile)));
                FrameArgs ap = a;
                ap.views = c->d_views.p + r->slot;
                ap.n_views = 1;
                ap.total_tiles = r->tiles;
                ap.view_offset = r->slot;
                ap.tile_offset = r->tiles_started;
                // the primary pass takes each new path's first shading step
                // (as a plain frame's does): survivors join the queue this
                // step's shade pass writes (live[(ps + 1) & 1], count at
                // CNT_LIVE + ps + 1) and their rays this step's trace pass
                // (CNT_RAY + ps); k_primary appends relative to the counters
                // it is given
                ap.counters = c->counters.p + ps;
                ap.live[1] = ((ps + 1u) & 1u) ? c->live1.p : c->live0.p;
                k_primary<false, true, 0><<<n, 256, 0, st>>>(ap);
                r->tiles_started += n;
                budget -= std::min<uint64_t>(budget, uint64_t(n) * per_tile);
            }
        }
        // 2. one shade + one trace pass over every live path
        k_shade<0><<<c->grid_shade, 256, 0, st>>>(a, ps);
        k_trace<false><<<c->grid_trace, 256, 0, st>>>(a, ps);
        if (ps == kRing - 1)  // wrap: the survivors' count moves to slot 0
            cudaMemcpyAsync(c->counters.p + CNT_LIVE, c->counters.p + CNT_LIVE + kRing, 4, cudaMemcpyDeviceToDevice,
                            st);
        s->step++;
        // 3. completion: remaining path counts per slot
        cudaMemcpyAsync(s->h_remaining, s->d_remaining, sizeof(uint32_t) * s->cfg.max_requests,
                        cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(s->h_stats, c->stats.p, sizeof(unsigned long long) * ST_TOTAL, cudaMemcpyDeviceToHost, st);
        const cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            serve_fail(s, VE_ERR_CUDA, std::string("serve step: ") + cudaGetErrorString(e));
            return;
        }
        std::vector<ServeRequest*> finished;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->rays = s->h_stats[ST_RAYS_PRIMARY] + s->h_stats[ST_RAYS_BOUNCE] + s->h_stats[ST_RAYS_SHADOW];
            s->steps_run++;
            for (ServeRequest* r : run) {
                if (r->tiles_started == r->tiles && s->h_remaining[r->slot] == 0) {
                    r->state = 2;
                    finished.push_back(r);
                }
            }
        }
        // resolves on the render stream (before the next step's passes);
        // the copies on the copy stream, overlapping the next steps
        for (ServeRequest* r : finished) {
            FrameArgs ar = a;
            ar.views = c->d_views.p + r->slot;
            ar.n_views = 1;
            ar.total_tiles = r->tiles;
            k_resolve<<<r->tiles, 256, 0, st>>>(ar);
        }
        if (!finished.empty()) {
            cudaEventRecord(s->resolve_ev, st);
            cudaStreamWaitEvent(s->copy_st, s->resolve_ev, 0);
            for (ServeRequest* r : finished) {
                const uint64_t np = r->pixels;
                if (r->out_vid)
                    cudaMemcpyAsync(r->out_vid, c->out_vid.p + r->pix_off, np * 4, cudaMemcpyDeviceToHost, s->copy_st);
                if (r->out_rgb)
                    cudaMemcpyAsync(r->out_rgb, c->out_rgb.p + 3 * r->pix_off, np * 12, cudaMemcpyDeviceToHost,
                                    s->copy_st);
                cudaEventRecord(r->done_ev, s->copy_st);
                cudaLaunchHostFunc(s->copy_st, serve_copied, r);
            }
        }
    }
}

}  // namespace ve

extern "C" {

int ve_server_create(ve_ctx* c, const ve_server_config* cfg, ve_server** out) {
    if (c) ve::join_alt(c);  // after the second frame set's frames in flight
    using namespace ve;
    if (!c || !cfg || !out) return fail(VE_ERR_INVALID, "server_create: null argument");
    if (cfg->max_requests == 0 || cfg->max_requests > 4096)
        return fail(VE_ERR_INVALID, "server_create: max_requests must be in [1, 4096]");
    if (cfg->pixel_capacity == 0 || cfg->path_capacity == 0 || cfg->path_capacity >= (1ull << 30) ||
        cfg->pixel_capacity >= (1ull << 32))
        return fail(VE_ERR_INVALID, "server_create: bad pool capacities");
    cudaSetDevice(c->device);
    int rc = ensure_frame(c, cfg->pixel_capacity, cfg->path_capacity, cfg->max_requests);
    if (rc) return rc;
    if ((rc = sync_scenes(c))) return rc;
    ve_server* s = new ve_server();
    s->c = c;
    s->cfg = *cfg;
    s->pix_pool.reset(cfg->pixel_capacity);
    s->path_pool.reset(cfg->path_capacity);
    for (uint32_t i = cfg->max_requests; i-- > 0;) s->free_slots.push_back(i);
    if (cudaMalloc(&s->d_remaining, 4ull * cfg->max_requests) != cudaSuccess ||
        cudaMallocHost(&s->h_remaining, 4ull * cfg->max_requests) != cudaSuccess ||
        cudaMallocHost(&s->h_view, sizeof(DevView) * cfg->max_requests) != cudaSuccess ||
        cudaMallocHost(&s->h_stats, sizeof(unsigned long long) * ST_TOTAL) != cudaSuccess ||
        cudaStreamCreateWithFlags(&s->copy_st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->resolve_ev, cudaEventDisableTiming) != cudaSuccess) {
        ve_server_destroy(s);
        return fail(VE_ERR_NOMEM, "server_create: allocation failed");
    }
    cudaMemsetAsync(s->d_remaining, 0, 4ull * cfg->max_requests, c->stream);
    cudaMemsetAsync(c->counters.p, 0, CNT_TOTAL * 4, c->stream);
    cudaMemsetAsync(c->stats.p, 0, ST_TOTAL * 8, c->stream);
    VE_CUDA(cudaStreamSynchronize(c->stream));
    s->worker = std::thread(serve_loop, s);
    *out = s;
    return VE_OK;
}

int ve_server_submit(ve_server* s, const ve_view* v, uint32_t* voxel_id_out, float* rgb_out, uint64_t* request_id) {
    using namespace ve;
    if (!s || !v || !request_id) return fail(VE_ERR_INVALID, "server_submit: null argument");
    const ve_frame_config& f = v->frame;
    if (v->scene_id < 0 || size_t(v->scene_id) >= s->c->scenes.size() || !s->c->scenes[v->scene_id].live)
        return fail(VE_ERR_NOT_FOUND, "server_submit: unknown scene");
    if (f.width == 0 || f.height == 0 || f.width > 16384 || f.height > 16384 || f.spp == 0 || f.spp > 1024 ||
        f.bounces + 2 > kMaxPasses || f.primary_controlchecks > kMaxControlChecks ||
        f.bounce_controlchecks > kMaxControlChecks || f.render_type > VE_RENDER_VARIANCE ||
        f.reconstruction_radius > 64)
        return fail(VE_ERR_INVALID, "server_submit: frame configuration out of range");
    ServeRequest* r = new ServeRequest();
    r->owner = s;
    r->view = *v;
    r->out_vid = voxel_id_out;
    r->out_rgb = rgb_out;
    r->pixels = uint64_t(f.width) * f.height;
    r->paths = r->pixels * f.spp;
    r->tiles = ((f.width + 15) / 16) * ((f.height + 15) / 16);
    if (r->pixels > s->cfg.pixel_capacity || r->paths > s->cfg.path_capacity) {
        delete r;
        return fail(VE_ERR_CAPACITY, "server_submit: request larger than the server's pools");
    }
    cudaSetDevice(s->c->device);
    cudaEventCreateWithFlags(&r->done_ev, cudaEventDisableTiming);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) {
            cudaEventDestroy(r->done_ev);
            delete r;
            return fail(s->error ? s->error : VE_ERR_STATE, "server_submit: server stopped: " + s->error_msg);
        }
        r->id = s->next_id++;
        r->t_submit = now_s();
        s->queue.push_back(r);
        s->all[r->id] = r;
    }
    s->cv_work.notify_one();
    *request_id = r->id;
    return VE_OK;
}

int ve_server_wait(ve_server* s, uint64_t id, uint32_t timeout_ms, ve_request_info* info) {
    using namespace ve;
    if (!s) return fail(VE_ERR_INVALID, "server_wait: null server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return fail(VE_ERR_NOT_FOUND, "server_wait: unknown request id");
    ServeRequest* r = it->second;
    const bool ok = s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms),
                                        [&] { return r->state == 3 || s->error != VE_OK; });
    if (s->error != VE_OK) return fail(s->error, "server_wait: " + s->error_msg);
    if (!ok) return fail(VE_ERR_TIMEOUT, "server_wait: request not finished within the timeout");
    if (info) {
        info->request_id = r->id;
        info->submit_s = r->t_submit;
        info->admit_s = r->t_admit;
        info->done_s = r->t_done;
        info->pixels = r->pixels;
        info->paths = r->paths;
    }
    cudaEventDestroy(r->done_ev);
    s->all.erase(it);
    delete r;
    return VE_OK;
}

int ve_server_get_stats(ve_server* s, ve_server_stats* out) {
    using namespace ve;
    if (!s || !out) return fail(VE_ERR_INVALID, "server_stats: null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    out->completed = s->completed;
    out->admitted = s->admitted;
    out->queued = s->queue.size();
    out->in_flight = s->active.size();
    out->max_in_flight = s->max_inflight;
    out->steps = s->steps_run;
    out->pool_bytes = s->pix_pool.capacity() * 48ull + s->path_pool.capacity() * 152ull;
    uint64_t scene_bytes = 0;
    for (const auto& sc : s->c->scenes)
        if (sc.live)
            scene_bytes += (sc.n_words + 8) * 4 + (sizeof(CacheEntry) << s->c->cfg.hash_log2) +
                           (sc.top_level ? (4ull << (3u * (sc.top_level - 1u))) : 0ull);
    out->scene_bytes = scene_bytes;
    out->rays = s->rays;
    return VE_OK;
}

int ve_server_destroy(ve_server* s) {
    if (!s) return VE_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    for (auto& kv : s->all) {
        if (kv.second->done_ev) cudaEventDestroy(kv.second->done_ev);
        delete kv.second;
    }
    if (s->d_remaining) cudaFree(s->d_remaining);
    if (s->h_remaining) cudaFreeHost(s->h_remaining);
    if (s->h_view) cudaFreeHost(s->h_view);
    if (s->h_stats) cudaFreeHost(s->h_stats);
    if (s->copy_st) {
        cudaStreamSynchronize(s->copy_st);
        cudaStreamDestroy(s->copy_st);
    }
    if (s->resolve_ev) cudaEventDestroy(s->resolve_ev);
    const int err = s->error;
    delete s;
    return err;
}

}  // extern "C"
