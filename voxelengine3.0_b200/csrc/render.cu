// render.cu — B200 wavefront renderer for the voxel ray pipeline and its
// C ABI (include/ve.h).
//
// Frame structure (the four passes of Renderer::runWavefrontFrame,
// reference src/renderer/renderer.cpp:282-649, in per-pixel form, with every
// host readback removed):
//   decay      radiance-cache temporal decay (once per scene per frame)
//   primary    one thread per pixel: camera ray + counted DDA -> GBuffer;
//              spp path states per hit pixel, appended to the live queue
//   shade/trace  bounce loop; shade consumes the live queue, adds the
//              pending sun-shadow result, shades the hit, emits the
//              extension ray and the sun shadow ray into one ray queue
//              (warp-ballot compaction) and deposits finished paths into the
//              radiance cache with warp-aggregated atomics (AccumPass);
//              trace runs the DDA for every queued ray
//   resolve    AvgPass + visualisation modes + ACES tonemap per pixel
// All queue sizes live in device counters: kernels size their loops from
// them, so a frame needs no host synchronisation.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ve.h"
#include "builder.cuh"
#include "emissive.cuh"
#include "lbuffer.cuh"
#include "nrc.cuh"
#include "raycast.cuh"
#include "ve_device.cuh"

namespace ve {
using namespace dev;

// ---------------------------------------------------------------------------
// device data
// ---------------------------------------------------------------------------
struct alignas(16) CacheEntry {
    uint32_t key;    // vid (voxelKey + 1); 0 = empty
    uint32_t count;  // exact number of deposits
    float l2;        // sum of luma^2 (decayed)
    uint32_t pad;
    float4 rgbw;     // sums of r, g, b and the decayed weight
};
static_assert(sizeof(CacheEntry) == 32, "cache entry is one 32-byte sector");

struct DevScene {
    const uint32_t* nodes;
    uint64_t n_words;
    CacheEntry* cache;
    uint32_t depth;
    uint32_t cache_log2;
    uint32_t probes;
    uint32_t top_level;   // T0: levels 0..T0-1 resolved by the top table (0: none)
    const uint32_t* top;  // top table, (2^(T0-1))^3 words
    // emissive lights (VE_FRAME_EMISSIVE; null until the scene's first such frame)
    EmLight* em_list;     // the registry, kEmCapacity records
    uint32_t* em_claim;   // claim table of registered (or dropped) light vids
    uint32_t* em_state;   // {registered lights, lights staged this frame}
    EmLight* em_stage;    // lights found this frame, appended at its end
    ResEntry* res;        // per-voxel ReSTIR reservoirs, 2^kResLog2 entries
    uint32_t* lbuf;       // the dual-channel lBuffer (VE_FRAME_LBUFFER; null until first used)
    const float4* ntab;   // ball-normal scenes: unit normal per code index (null: 3x3x3 gradient)
    uint32_t n_ntab;
    // the box of the cells that can hold a voxel, widened by one voxel on
    // every side (bounce rays end when they leave it; see k_trace)
    float clip_lo[3], clip_hi[3];
};

struct DevMaterial {
    float4 albedo_rough;  // albedo rgb, roughness
    float4 params;        // metallic, specular, emissive (0/1), emissive intensity
};

struct DevView {
    float cam[16];
    uint32_t scene, W, H, spp;
    uint32_t bounces, cc_primary, cc_bounce, recon_radius;
    uint32_t render_type, frame_index, flags, tiles_x;
    float sun[3], sun_intensity;
    float sky[3], decay;
    float variance_norm;
    uint32_t pix_base;
    uint32_t tile_base;
    uint32_t pad0;
    unsigned long long path_base;
    // importance-aware scheduling (rank.comp knobs)
    float w_pix, w_var, pix_norm, top_frac, mid_frac;
    uint32_t min_samples, budget, pad1;
    // emissive NEE / ReSTIR DI (core.hpp:138-144 knobs)
    uint32_t restir, restir_m, restir_nbrs, restir_max_m;
    float restir_radius;
    uint32_t pad2, pad3, pad4;
    // dual-channel lBuffer (core.hpp:93-104, 150-157 knobs)
    LbParams lb;
    uint32_t pad5;
    // rows whose paths start (split frames: the rank's band) and rows whose
    // primary rays run (the band and the AvgPass's halo); [0, H) otherwise
    uint32_t row_lo, row_hi, g_lo, g_hi;
};

enum : uint32_t { kMaxPasses = 18, kMaxControlChecks = 65536 };
constexpr uint32_t kDefaultRefill = 20;  // trace refill threshold (idle lanes of 32)
enum : uint32_t {
    CNT_LIVE = 0, CNT_RAY = 20, CNT_CURSOR = 40, CNT_NRC_Q = 60, CNT_NRC_S = 61, CNT_SCHED = 62, CNT_RES = 63,
    CNT_RAYSH = 64,  // shadow rays per pass (extension rays: CNT_RAY)
    CNT_TOTAL = 96
};
enum : uint32_t {
    ST_RAYS_PRIMARY = 0,
    ST_RAYS_BOUNCE,
    ST_RAYS_SHADOW,
    ST_FETCH,        // node words read by k_primary + k_trace
    ST_PATHS,
    ST_DEPOSITS,
    ST_DROPPED,
    ST_STEPS,        // DDA iterations of k_primary + k_trace
    ST_FETCH_TRACE,  // node words read by k_trace alone
    ST_STEPS_TRACE,
    ST_NRC_QUERIES,  // paths ended at their second vertex by the learned cache
    ST_NRC_HASH,     // ... by the hashed per-voxel cache
    ST_NRC_SAMPLES,  // training samples recorded
    ST_SCHED_VOXELS, // scheduled frames: distinct visible voxels
    ST_SCHED_PATHS,  // scheduled frames: shade-list entries
    ST_EM_LIGHTS,    // emissive frames: registered lights after the frame
    ST_EM_NEE,       // emissive frames: NEE shadow rays toward lights
    ST_RES_WRITES,   // emissive frames: reservoirs committed
    ST_SHADOW_SHARED,  // sun shadow rays answered by the same pixel's sample-0 traversal
    ST_TOTAL = 20
};
// path flags (meta.z bits 24-31); F_DZERO / F_IZERO: the path's direct /
// indirect radiance is +0 in every channel and its p_direct / p_indirect slot
// was not written (loads of the slot are discarded)
enum : uint32_t { F_PENDING = 1u, F_TERM = 2u, F_TRAIN = 4u, F_DZERO = 8u, F_IZERO = 16u };
__device__ __forceinline__ bool pos_zero(f3 v) {
    return (__float_as_uint(v.x) | __float_as_uint(v.y) | __float_as_uint(v.z)) == 0u;
}
// Shading-kernel instances: emissive NEE (VE_FRAME_EMISSIVE) and the
// dual-channel lBuffer AccumPass (VE_FRAME_LBUFFER) compile into their own
// instances so the plain kernels keep their registers.
// kModeNrc: the batch ends paths at their second vertex (VE_FRAME_LEARNED /
// _TERMINATE_HASH / _TRAIN); only the shade pass needs that instance, since
// the primary and scheduled-emit passes shade vertex 0 only.
constexpr int kModeEm = 1, kModeLb = 2, kModeNrc = 4;
// a cached voxel average ends a path (VE_FRAME_TERMINATE_HASH, and the
// learned cache's fallback) only when at least this many deposits made it
constexpr uint32_t kHashTermMinCount = 8;
// validation samples a cell needs before its error decides for or against the
// learned cache
constexpr uint32_t kMinCellSamples = 4;

struct FrameArgs {
    const DevView* views;
    uint32_t n_views;
    uint32_t total_tiles;
    const DevScene* scenes;
    const DevMaterial* mats;
    // path state (structure of arrays, index = global path id)
    float4* p_ray_o;     // next ray origin (shading point)
    float4* p_ray_d;     // direction of the ray that produced the current hit / next extension ray
    float4* p_tp;        // throughput
    float4* p_direct;    // direct radiance (sun at bounce 0, bounce-0 emission)
    float4* p_indirect;  // indirect radiance
    float4* p_pend;      // pending NEE contribution; w: the shadow trace's result code (~0 escaped, hit vid, 0)
    float4* p_sdir;      // emissive batches: NEE shadow direction, w = the light's vid (~0 for the sun)
    PathRes* p_res;      // emissive batches: a path's bounce-0 reservoir until the commit
    uint32_t* res_list;  // paths holding a reservoir (counter CNT_RES)
    LbRec* lb_rec;       // lBuffer frames: each path's deposit, at its path slot
    uint32_t* lb_key;    // ... and its lBuffer row (0: the path made no deposit)
    uint4* p_hit;        // {status, leaf word, x | y<<16, z | material<<16}
    uint4* p_meta;       // {vid, rng, view | bounce<<16 | flags<<24, pixel}
    uint32_t* live[2];
    // per pass: extension rays {path slot, view}, and shadow rays {path slot |
    // 1 << 31 (| 1 << 30: shared by the pixel's samples), view} in a separate
    // region; the view rides along so a trace refill needs no path-state load
    // before the ray's own
    uint2* rayq;
    uint2* rayq_sh;
    uint32_t* counters;
    unsigned long long* stats;
    uint4* gbuf;
    uint32_t* out_vid;
    uint32_t* out_node;
    float* out_rgb;
    float* out_mapped;
    uchar4* out_mapped8;  // the displayed RGBA8 image (final.frag into the framebuffer)
    float* path_rgb;
    uint32_t refill;       // idle lanes at which a trace warp takes new rays
    uint32_t view_offset;  // index of views[0] in the view table the paths refer to
    uint32_t tile_offset;  // primary pass: block b covers tile b + tile_offset (serving spreads a request's tiles)
    uint32_t* remaining;   // per view slot: paths not yet deposited (serving), or null
    // learned radiance cache (views with VE_FRAME_LEARNED / _TERMINATE_HASH / _TRAIN)
    nrc::QRec* nq;         // queries: paths ended at their second vertex by the network
    float4* nstage;        // per query: {tp, path}, {direct, vid}, {indirect, scene | path-rgb flag}
    nrc::QRec* ns;         // training sample inputs
    nrc::TRec* nt;         // training sample targets
    uint32_t nq_cap, ns_cap;
    uint32_t train_thresh;  // a path is a training path when hash(path, frame) < this
    float fallback_thr;     // per-cell validation error above which the hash cache answers
    const float4* val;      // per cell: {mean target, samples}, {mean prediction}
    uint32_t val_mask;
    uint32_t nrc_ready;     // cells without validation samples use the network
    uint32_t* p_aux;        // per path: training sample slot
    // importance-aware scheduling (VE_FRAME_SCHEDULED, single view)
    uint4* hitinfo;         // per pixel: {leaf word, x | y << 16, z | material << 16, 0} of the primary hit
    uint32_t* claim_key;    // per-frame voxel claim table (vid, 0 = free)
    uint32_t* claim_pix;    // canonical (smallest) pixel of the voxel
    uint32_t* claim_cnt;    // pixels that see the voxel
    uint32_t claim_mask;
    uint32_t* sched_n;      // per pixel: paths of its voxel when it is the canonical pixel
    uint32_t* sched_off;    // exclusive prefix sum of sched_n
    uint2* shade_list;      // {vid, pixel} per path
    uint32_t shade_cap;
    float* rank;            // the scene's {t_high, t_mid, histogram[256]} (thresholds from the previous frame)
};

constexpr uint32_t kRankBins = 256;
constexpr uint32_t kClaimProbes = 64;

// ---------------------------------------------------------------------------
// warp helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

// Warp-aggregated queue append: one atomicAdd per warp; returns this lane's
// slot.  Must be called by all 32 lanes.
__device__ __forceinline__ uint32_t warp_append(bool pred, uint32_t* counter, uint32_t per_lane = 1u) {
    const unsigned m = __ballot_sync(0xffffffffu, pred);
    if (m == 0u) return 0u;
    const uint32_t lane = lane_id();
    const int leader = __ffs(m) - 1;
    uint32_t base = 0;
    if (int(lane) == leader) base = atomicAdd(counter, uint32_t(__popc(m)) * per_lane);
    base = __shfl_sync(0xffffffffu, base, leader);
    return base + uint32_t(__popc(m & ((1u << lane) - 1u))) * per_lane;
}

__device__ __forceinline__ void warp_add_stat(unsigned long long* stat, uint32_t v) {
    uint32_t s = v;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane_id() == 0 && s) atomicAdd(stat, (unsigned long long)s);
}

// Radiance cache: power-of-two table, Fibonacci hash of the vid, linear
// probing, claim by CAS on the key.
__device__ __forceinline__ uint32_t cache_home(uint32_t vid, uint32_t log2n) {
    return (vid * 0x9E3779B1u) >> (32u - log2n);
}
__device__ __forceinline__ int cache_claim(CacheEntry* c, uint32_t log2n, uint32_t probes, uint32_t vid) {
    const uint32_t mask = (1u << log2n) - 1u;
    const uint32_t h = cache_home(vid, log2n);
    for (uint32_t i = 0; i < probes; i++) {
        const uint32_t s = (h + i) & mask;
        uint32_t k = *((volatile uint32_t*)&c[s].key);
        if (k == vid) return int(s);
        if (k == 0u) {
            k = atomicCAS(&c[s].key, 0u, vid);
            if (k == 0u || k == vid) return int(s);
        }
    }
    return -1;
}
__device__ __forceinline__ int cache_find(const CacheEntry* c, uint32_t log2n, uint32_t probes, uint32_t vid) {
    const uint32_t mask = (1u << log2n) - 1u;
    const uint32_t h = cache_home(vid, log2n);
    for (uint32_t i = 0; i < probes; i++) {
        const uint32_t s = (h + i) & mask;
        const uint32_t k = c[s].key;
        if (k == vid) return int(s);
        if (k == 0u) return -1;
    }
    return -1;
}

struct DepSlot {
    float r, g, b, l2;
};

// AccumPass deposit, warp-aggregated: lanes depositing into the same
// (scene, vid) are merged in shared memory and one leader lane issues the
// atomics (count, luma^2, and one vector add of {r, g, b, weight}).
// `n_dep` / `n_drop`: this thread's share of the deposits made / dropped
// (a group's leader counts the group), added to the frame's counters once
// per kernel instead of by one atomic per group on a single address.
__device__ __forceinline__ void warp_deposit(bool active, uint32_t scene, uint32_t vid, float r, float g, float b,
                                             float l2, DepSlot* sh, const DevScene* scenes, uint32_t& n_dep,
                                             uint32_t& n_drop) {
    const unsigned am = __ballot_sync(0xffffffffu, active);
    if (am == 0u) return;
    const uint32_t lane = lane_id();
    if (active) sh[lane] = DepSlot{r, g, b, l2};
    __syncwarp();
    if (active) {
        const unsigned long long key = (static_cast<unsigned long long>(scene) << 32) | vid;
        const unsigned peers = __match_any_sync(am, key);
        if (int(lane) == __ffs(peers) - 1) {
            float sr = 0.0f, sg = 0.0f, sb = 0.0f, sl = 0.0f;
            for (unsigned m = peers; m; m &= m - 1u) {
                const int j = __ffs(m) - 1;
                sr += sh[j].r;
                sg += sh[j].g;
                sb += sh[j].b;
                sl += sh[j].l2;
            }
            const uint32_t n = uint32_t(__popc(peers));
            const DevScene& S = scenes[scene];
            const int s = cache_claim(S.cache, S.cache_log2, S.probes, vid);
            if (s >= 0) {
                CacheEntry* e = S.cache + s;
                atomicAdd(&e->count, n);
                atomicAdd(&e->l2, sl);
                atomicAdd(&e->rgbw, make_float4(sr, sg, sb, float(n)));
                n_dep += n;
            } else {
                n_drop += n;
            }
        }
    }
    __syncwarp();
}

// Per-thread tallies of a shading kernel, added to the frame's counters once
// at its end.
struct EmitCounts {
    uint32_t ext = 0, sh = 0, dep = 0, drop = 0, shared = 0;
};
__device__ __forceinline__ void flush_counts(const EmitCounts& c, unsigned long long* stats) {
    warp_add_stat(&stats[ST_RAYS_BOUNCE], c.ext);
    warp_add_stat(&stats[ST_RAYS_SHADOW], c.sh);
    warp_add_stat(&stats[ST_SHADOW_SHARED], c.shared);
    warp_add_stat(&stats[ST_DEPOSITS], c.dep);
    warp_add_stat(&stats[ST_DROPPED], c.drop);
}

// Block-aggregated appends to a shading step's three queues (live paths,
// extension rays, shadow rays): one atomicAdd per queue and block instead of
// per warp — each queue counter is a single address every block contends
// on.  Called by all threads of a block of <= 256; successive calls
// alternate between two buffers, so one barrier pair per call suffices.
struct BlockQ {
    uint32_t cnt[3][8];
    uint32_t base[3];
};
__device__ __forceinline__ uint3 block_append3(bool p0, bool p1, bool p2, uint32_t* c0, uint32_t* c1, uint32_t* c2,
                                               BlockQ& q) {
    const uint32_t lane = lane_id(), w = threadIdx.x >> 5;
    const unsigned m0 = __ballot_sync(0xffffffffu, p0);
    const unsigned m1 = __ballot_sync(0xffffffffu, p1);
    const unsigned m2 = __ballot_sync(0xffffffffu, p2);
    if (lane == 0u) {
        q.cnt[0][w] = uint32_t(__popc(m0));
        q.cnt[1][w] = uint32_t(__popc(m1));
        q.cnt[2][w] = uint32_t(__popc(m2));
    }
    __syncthreads();
    if (threadIdx.x < 3u) {
        const uint32_t k = threadIdx.x;
        uint32_t acc = 0;
        for (uint32_t i = 0; i < (blockDim.x >> 5); i++) {
            const uint32_t c = q.cnt[k][i];
            q.cnt[k][i] = acc;
            acc += c;
        }
        uint32_t* ctr = k == 0u ? c0 : (k == 1u ? c1 : c2);
        q.base[k] = acc ? atomicAdd(ctr, acc) : 0u;
    }
    __syncthreads();
    const unsigned lt = (1u << lane) - 1u;
    return make_uint3(q.base[0] + q.cnt[0][w] + uint32_t(__popc(m0 & lt)),
                      q.base[1] + q.cnt[1][w] + uint32_t(__popc(m1 & lt)),
                      q.base[2] + q.cnt[2][w] + uint32_t(__popc(m2 & lt)));
}

__device__ __forceinline__ uint32_t find_view(const DevView* views, uint32_t n, uint32_t tile) {
    uint32_t lo = 0, hi = n;  // last view with tile_base <= tile
    while (hi - lo > 1u) {
        const uint32_t mid = (lo + hi) >> 1;
        if (views[mid].tile_base <= tile) lo = mid; else hi = mid;
    }
    return lo;
}

// 16x16 pixel tile per 256-thread block; each warp covers an 8x4 sub-tile.
__device__ __forceinline__ void tile_pixel(uint32_t local_tile, uint32_t tiles_x, uint32_t* px, uint32_t* py) {
    const uint32_t w = threadIdx.x >> 5, l = threadIdx.x & 31u;
    *px = (local_tile % tiles_x) * 16u + (w & 1u) * 8u + (l & 7u);
    *py = (local_tile / tiles_x) * 16u + (w >> 1) * 4u + (l >> 3);
}

__device__ __forceinline__ f3 ld3(const float4& v) { return mk(v.x, v.y, v.z); }
__device__ __forceinline__ float4 st3(f3 v, float w = 0.0f) { return make_float4(v.x, v.y, v.z, w); }

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------

// Radiance-cache temporal decay: sums and weight *= decay (counts exact).
__global__ void __launch_bounds__(256) k_decay(CacheEntry* cache, uint32_t n, float decay) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (cache[i].key == 0u) continue;
        float4 v = cache[i].rgbw;
        v.x = v.x * decay; v.y = v.y * decay; v.z = v.z * decay; v.w = v.w * decay;
        cache[i].rgbw = v;
        cache[i].l2 = cache[i].l2 * decay;
    }
}

// trace.comp:25-70 for extension rays; shadow rays test escape toward the sun.
//
// Persistent kernel with per-lane refill: a lane whose ray has finished takes
// the next queue entry (one warp-aggregated atomicAdd on a per-pass cursor
// serves all idle lanes of the warp, once `refill` of them are idle or none is
// busy), so warps stay full although ray lengths differ by 100x.  One ballot
// per step: once a refill hands out the queue's last entry the warp stops
// refilling (a warp-uniform flag) and runs its remaining rays out.
// EM: the batch has VE_FRAME_EMISSIVE views (shadow rays toward lights).
// FLAT: every scene of the batch has a top table reaching its leaves
// (T0 = D): the descent keeps one leaf-block offset instead of the per-level
// array (dda_step).
template <bool COUNT, bool EM = false, bool FLAT = false>
__global__ void __launch_bounds__(256, 6) k_trace(FrameArgs a, uint32_t pass) {
    // the pass's extension rays, then its shadow rays: warps stay mostly of
    // one kind, and the shorter shadow rays form the tail of the pass
    const uint32_t n_ext = a.counters[CNT_RAY + pass];
    const uint32_t n = n_ext + a.counters[CNT_RAYSH + pass];
    uint32_t* cursor = &a.counters[CNT_CURSOR + pass];
    const uint32_t lane = lane_id();
    bool active = false;
    bool drained = false;  // warp-uniform: every ray of the pass has been handed out
    uint32_t e = 0, D = 0, T0 = 0;
    const uint32_t* nodes = nullptr;
    const uint32_t* top = nullptr;
    uint32_t n_words = 0;
    Dda s;
    RayCount rc;
    for (;;) {
        // the result lives one iteration: written and stored when a ray ends
        Hit h;
        h.status = kEscaped;
        h.id = h.material = h.x = h.y = h.z = 0u;
        const unsigned busy = __ballot_sync(0xffffffffu, active);
        if (drained && busy == 0u) break;
        const unsigned idle = drained ? 0u : ~busy;
        bool finished = false;
        if (idle != 0u && (uint32_t(__popc(idle)) >= a.refill || busy == 0u)) {
            const int leader = __ffs(idle) - 1;
            uint32_t first_idx = 0;
            if (int(lane) == leader) first_idx = atomicAdd(cursor, uint32_t(__popc(idle)));
            first_idx = __shfl_sync(0xffffffffu, first_idx, leader);
            drained = first_idx + uint32_t(__popc(idle)) >= n;
            if (!active) {
                const uint32_t idx = first_idx + uint32_t(__popc(idle & ((1u << lane) - 1u)));
                if (idx < n) {
                    const uint2 en = idx < n_ext ? a.rayq[idx] : a.rayq_sh[idx - n_ext];
                    e = en.x;
                    const uint32_t p = e & 0x3FFFFFFFu;
                    const DevView& v = a.views[en.y];
                    const DevScene S = a.scenes[v.scene];
                    nodes = S.nodes;
                    n_words = word_bound(S.n_words);
                    D = S.depth;
                    top = S.top;
                    T0 = S.top_level;
                    const f3 o = ld3(a.p_ray_o[p]);
                    f3 d = (e >> 31) ? mk(v.sun[0], v.sun[1], v.sun[2]) : ld3(a.p_ray_d[p]);
                    if (EM && (e >> 31) && (v.flags & VE_FRAME_EMISSIVE)) d = ld3(a.p_sdir[p]);
                    finished = dda_init(s, o, d, v.cc_bounce, D, h);
                    {
                        // a bounce ray that escapes or times out shades as
                        // sky alike, so it ends on leaving the box of the
                        // cells that can hold a voxel (exit of its slab);
                        // shadow rays walk on (there a timeout is a shadow).
                        // Fetch-counting frames count this walk too.
                        float te = __int_as_float(0x7f800000);
                        if (!(e >> 31)) {
                            const float tx = ((s.inv.x > 0.0f ? S.clip_hi[0] : S.clip_lo[0]) - s.o.x) * s.inv.x;
                            const float ty = ((s.inv.y > 0.0f ? S.clip_hi[1] : S.clip_lo[1]) - s.o.y) * s.inv.y;
                            const float tz = ((s.inv.z > 0.0f ? S.clip_hi[2] : S.clip_lo[2]) - s.o.z) * s.inv.z;
                            te = gmin(gmin(tx, ty), tz);
                        }
                        s.t_end = te;
                    }
                    active = !finished;
                }
            }
        }
        if (active) {
            finished = dda_step<COUNT, true, true, FLAT && !COUNT>(s, nodes, n_words, D, top, T0, h, rc);
            if (finished) active = false;
        }
        if (finished) {
            const uint32_t p = e & 0x3FFFFFFFu;
            if (e >> 31) {
                // the shadow ray's result code: ~0 left the volume, a hit
                // voxel's vid (emissive batches: the light must be the hit),
                // else 0 (the record's initial value).  A shared sun shadow
                // ray (bit 30: a pixel's samples start at the same hit) finds
                // in its record the count of the records that follow it and
                // take the same code.
                uint32_t* rec = reinterpret_cast<uint32_t*>(a.p_pend + p) + 3;
                if (!EM && (e & 0x40000000u)) {
                    const uint32_t n = *rec, code = h.status == kEscaped ? 0xFFFFFFFFu : 0u;
                    for (uint32_t k = 0; k <= n; k++) rec[4u * k] = code;
                } else if (h.status == kEscaped) {
                    *rec = 0xFFFFFFFFu;
                } else if (EM && h.status == kHit) {
                    *rec = voxel_key(h.x, h.y, h.z) + 1u;
                }
            } else {
                // h.id holds the hit leaf's word: the shade pass needs no
                // dependent load from the node array
                a.p_hit[p] = make_uint4(h.status, h.id, h.x | (h.y << 16), h.z | (h.material << 16));
            }
        }
    }
    if (COUNT) {
        warp_add_stat(&a.stats[ST_FETCH], rc.fetch);
        warp_add_stat(&a.stats[ST_STEPS], rc.steps);
        warp_add_stat(&a.stats[ST_FETCH_TRACE], rc.fetch);
        warp_add_stat(&a.stats[ST_STEPS_TRACE], rc.steps);
    }
}

// Adds the frame's counters to the running totals (ve_get_total_stats).
__global__ void k_accum_stats(const unsigned long long* frame, unsigned long long* total) {
    if (threadIdx.x < ST_TOTAL) total[threadIdx.x] += frame[threadIdx.x];
}

struct Avg {
    f3 rgb;
    uint32_t count;
    float var;
};
// lookupVoxelAvg (resolve.comp:109-148) over the FP32 cache
__device__ __forceinline__ Avg lookup_avg(const DevScene& S, uint32_t vid) {
    Avg r{mk(0.0f, 0.0f, 0.0f), 0u, 0.0f};
    if (vid == 0u) return r;
    const int s = cache_find(S.cache, S.cache_log2, S.probes, vid);
    if (s < 0) return r;
    const CacheEntry& e = S.cache[s];
    r.count = e.count;
    const float4 v = e.rgbw;
    if (r.count == 0u || !(v.w > 0.0f)) return r;
    const float inv = 1.0f / v.w;
    r.rgb = mk(v.x * inv, v.y * inv, v.z * inv);
    const float meanL = ((v.x + v.y) + v.z) * inv / 3.0f;
    r.var = gmax(e.l2 * inv - meanL * meanL, 0.0f);
    return r;
}

// The view's radiance cache: the dual-channel lBuffer (VE_FRAME_LBUFFER) or
// the FP32 per-voxel cache.
template <bool LB>
__device__ __forceinline__ Avg lookup_view(const DevView& v, const DevScene& S, uint32_t vid) {
    if (LB && (v.flags & VE_FRAME_LBUFFER) && S.lbuf) {
        Avg r;
        lb_lookup(S.lbuf, vid, r.rgb, r.count, r.var);
        return r;
    }
    return lookup_avg(S, vid);
}

// Octahedral map of a unit vector to [-1, 1]^2 (Cigolle et al. 2014): the
// learned cache's normal and direction inputs.
__device__ __forceinline__ float2 oct_encode(f3 v) {
    const float sum = (fabsf(v.x) + fabsf(v.y)) + fabsf(v.z);
    float x = v.x / sum, y = v.y / sum;
    if (v.z < 0.0f) {
        const float ox = (1.0f - fabsf(y)) * (x >= 0.0f ? 1.0f : -1.0f);
        const float oy = (1.0f - fabsf(x)) * (y >= 0.0f ? 1.0f : -1.0f);
        x = ox;
        y = oy;
    }
    return make_float2(x, y);
}

// packRgbL2 clamp (shade.comp:154-160): the deposited value is the clamped
// direct plus the clamped indirect radiance; NaN counts as zero.
__device__ __forceinline__ void deposit_value(f3 direct, f3 indirect, float& r, float& g, float& b, float& l2) {
    const float dv[3] = {direct.x, direct.y, direct.z};
    const float iv[3] = {indirect.x, indirect.y, indirect.z};
    float outv[3];
    for (int c = 0; c < 3; c++) {
        float x = dv[c], y = iv[c];
        if (!(x == x)) x = 0.0f;
        if (!(y == y)) y = 0.0f;
        outv[c] = gclamp(x, 0.0f, 1024.0f) + gclamp(y, 0.0f, 1024.0f);
    }
    r = outv[0];
    g = outv[1];
    b = outv[2];
    const float Lf = ((r + g) + b) / 3.0f;
    l2 = Lf * Lf;
}

// Training target of a finished training path: the radiance it gathered
// from its second vertex on, divided by the throughput it arrived there with.
__device__ __forceinline__ void write_target(nrc::TRec* t, f3 total, f3 s, f3 tp) {
    const f3 d = mk((total.x - s.x) / tp.x, (total.y - s.y) / tp.y, (total.z - s.z) / tp.z);
    const bool ok = tp.x > 0.0f && tp.y > 0.0f && tp.z > 0.0f && isfinite(d.x) && isfinite(d.y) && isfinite(d.z);
    t->tr = d.x;
    t->tg = d.y;
    t->tb = d.z;
    t->valid = ok ? 1u : 0u;
}

// Per-path result of one shading step, consumed by the warp-collective
// appends and deposits of the calling kernel.
struct ShadeOut {
    bool do_dep = false, app_live = false, app_ext = false, app_sh = false;
    // learned cache: a query (its record parked in the path's ray slots until
    // the warp's append), a recorded training sample, a hash-cache ending
    bool want_q = false, sampled = false, hash_term = false;
    bool app_res = false, em_nee = false;  // a reservoir to commit; an emissive NEE shadow ray
    bool sh_shared = false;  // a sun shadow ray traced by the pixel's sample-0 path instead
    bool sh_owner = false;   // ... the sample-0 path's ray, whose result the others take
    float dr = 0.0f, dg = 0.0f, db = 0.0f, dl2 = 0.0f;
    float ir = 0.0f, ig = 0.0f, ib = 0.0f;  // lBuffer frames: dr..db direct, ir..ib indirect
    uint32_t dvid = 0, dscene = 0, dview = 0;
};

__device__ __forceinline__ f3 clamp_contrib(f3 c) {
    return mk(gmin(c.x, kMaxContrib), gmin(c.y, kMaxContrib), gmin(c.z, kMaxContrib));
}

// A NEE sample waiting for its shadow ray: the contribution (already times
// the throughput) and the ray toward the light voxel `target`.
__device__ __forceinline__ void nee_pending(const FrameArgs& a, uint32_t p, f3 contrib, f3 ld, uint32_t target,
                                            uint32_t& nf, ShadeOut& o) {
    a.p_pend[p] = st3(contrib, 0.0f);
    a.p_sdir[p] = make_float4(ld.x, ld.y, ld.z, __uint_as_float(target));
    nf |= F_PENDING;
    o.app_sh = true;
    o.em_nee = true;
}

// Next-event estimation toward the registered emissive voxels at a
// non-emissive hit of bounce b < 2 (shade.comp:615-836): ReSTIR DI at
// bounce 0 when enabled (initial RIS over restir_m uniform candidates,
// temporal reuse of the voxel's reservoir, spatial reuse of neighbours',
// one shadow ray on the chosen sample), else the single-pick RIS estimator
// (4 power-weighted candidates, a uniform point on a uniform face).
// `rng` continues the path's sequence; the bounce sampling draws after it.
__device__ __forceinline__ void emissive_nee(const FrameArgs& a, const DevView& v, const DevScene& S, uint32_t p,
                                             uint32_t primary_vid, uint32_t b, uint32_t hx, uint32_t hy, uint32_t hz,
                                             f3 N, f3 sp, f3 dir, f3 tp, f3 albedo, float roughness, float metallic,
                                             float spec, uint32_t& rng, uint32_t& nf, ShadeOut& o) {
    const uint32_t n_lights = min(S.em_state[0], kEmCapacity);
    if (n_lights == 0u) return;  // frame-0 pre-discovery
    const EmLight* lights = S.em_list;
    if ((v.restir & VE_RESTIR_ENABLE) && b == 0u) {
        Reservoir res{0u, 0u, 0u, 0.0f, 0u, 0.0f};
        // (1) initial RIS, source pdf 1 / (lights x 6 faces)
        const uint32_t n_m = max(v.restir_m, 1u);
        const float inv_src = float(n_lights) * 6.0f;
        for (uint32_t k = 0; k < n_m; k++) {
            uint32_t pick = uint32_t(rand01(rng) * float(n_lights));
            if (pick >= n_lights) pick = n_lights - 1u;
            const EmLight cand = lights[pick];
            uint32_t face = uint32_t(rand01(rng) * 6.0f);
            if (face >= 6u) face = 5u;
            const float uu = rand01(rng);
            const float vv = rand01(rng);
            const uint32_t seed = pack_face_seed(face, uu, vv);
            const float target = target_pdf(cand, seed, sp, N);
            r_update(res, pick, cand.vid, seed, target, target * inv_src, rng);
        }
        // (2) temporal reuse: the voxel's committed reservoir
        if (v.restir & VE_RESTIR_TEMPORAL) {
            Reservoir t;
            if (res_load(S.res, primary_vid, lights, n_lights, t)) {
                r_cap(t, v.restir_max_m);
                r_combine(res, t, t.target, rng);
            }
        }
        // (3) spatial reuse: neighbour voxels in the surface's tangent plane
        if ((v.restir & VE_RESTIR_SPATIAL) && v.restir_nbrs > 0u) {
            const f3 up = fabsf(N.z) < 0.999f ? mk(0.0f, 0.0f, 1.0f) : mk(1.0f, 0.0f, 0.0f);
            const f3 T = normalize(cross(up, N));
            const f3 B = cross(N, T);
            const uint32_t K = min(v.restir_nbrs, 6u);
            for (uint32_t k = 0; k < K; k++) {
                const float ua = rand01(rng);
                const float rr = v.restir_radius * sqrtf(rand01(rng));
                float sn, cs;
                sincos_turn(ua, &sn, &cs);
                const f3 off = muls(add(muls(T, cs), muls(B, sn)), rr);
                const int ox = int(roundf(off.x)), oy = int(roundf(off.y)), oz = int(roundf(off.z));
                if (ox == 0 && oy == 0 && oz == 0) continue;
                const uint32_t nvid = neighbour_vid(hx, hy, hz, 1u, ox, oy, oz);
                if (nvid == 0u || nvid == primary_vid) continue;
                Reservoir nb;
                if (!res_load(S.res, nvid, lights, n_lights, nb)) continue;
                const float tu = target_pdf(lights[nb.light_idx], nb.seed, sp, N);
                if (tu <= 0.0f) continue;
                r_cap(nb, v.restir_max_m);
                r_combine(res, nb, tu, rng);
            }
        }
        // (4) one shadow ray on the chosen sample; contribution f W with the
        // size^2 Jacobian of the (face, u, v) parameterisation
        if (res.m > 0u && res.target > 0.0f) {
            const EmLight L = lights[res.light_idx];
            if (L.vid == res.light_vid) {
                f3 P, LN;
                light_sample_point(res.seed, L, P, LN);
                const f3 to = sub(P, sp);
                const float d2 = dot(to, to);
                const float dist = sqrtf(gmax(d2, 1e-12f));
                if (dist > 1e-3f) {
                    const f3 ld = divs(to, dist);
                    const float cx = gmax(dot(N, ld), 0.0f);
                    const float cy = gmax(dot(mk(-ld.x, -ld.y, -ld.z), LN), 0.0f);
                    if (cx > 0.0f && cy > 0.0f) {
                        const f3 brdf = evaluate_brdf(dir, ld, N, albedo, roughness, metallic, spec);
                        const float W = res.wsum / (float(res.m) * res.target);
                        const float sz2 = float(L.size * L.size);
                        const float geom = cy / gmax(d2, 1e-6f);
                        const f3 c = clamp_contrib(muls(muls(muls(mul(mk(L.er, L.eg, L.eb), brdf), geom), sz2), W));
                        nee_pending(a, p, mul(tp, c), ld, L.vid, nf, o);
                    }
                }
            }
        }
        // (5) the reservoir competes for the voxel's slot (committed at frame end)
        if (res.m > 0u) {
            const int e = res_claim(S.res, primary_vid);
            if (e >= 0) {
                atomicMax(&S.res[e].winner, p + 1u);
                a.p_res[p] = PathRes{uint32_t(e), res, v.scene};
                o.app_res = true;
            }
        }
        return;
    }
    // single-pick RIS NEE
    float wsum = 0.0f, chosen_t = 0.0f;
    uint32_t chosen = 0u;
    for (int k = 0; k < 4; k++) {
        uint32_t pick = uint32_t(rand01(rng) * float(n_lights));
        if (pick >= n_lights) pick = n_lights - 1u;
        const EmLight cand = lights[pick];
        const float lum = gmax(luminance(cand.er, cand.eg, cand.eb), 1e-6f);
        const float target = lum * float(cand.size * cand.size);
        wsum += target;
        if (rand01(rng) * wsum < target) {
            chosen = pick;
            chosen_t = target;
        }
    }
    const float avg_t = wsum / 4.0f;
    const EmLight L = lights[chosen];
    uint32_t face = uint32_t(rand01(rng) * 6.0f);
    if (face >= 6u) face = 5u;
    f3 fn, ft, fb;
    face_frame(face, fn, ft, fb);
    const float u1 = rand01(rng);
    const float u2 = rand01(rng);
    const f3 lp = face_point(L, fn, ft, fb, u1, u2);
    f3 ld = sub(lp, sp);
    const float d2 = dot(ld, ld);
    const float dist = sqrtf(d2);
    if (dist > 1e-3f && chosen_t > 0.0f) {
        ld = divs(ld, dist);
        const float cx = gmax(dot(N, ld), 0.0f);
        const float cy = gmax(dot(mk(-ld.x, -ld.y, -ld.z), fn), 0.0f);
        if (cx > 0.0f && cy > 0.0f) {
            const f3 brdf = evaluate_brdf(dir, ld, N, albedo, roughness, metallic, spec);
            const float area = 6.0f * float(L.size) * float(L.size);
            const float ris = float(n_lights) * avg_t / gmax(chosen_t, 1e-6f);
            const float geom = cy / gmax(d2, 1e-6f);
            const f3 c = clamp_contrib(muls(muls(muls(mul(mk(L.er, L.eg, L.eb), brdf), geom), area), ris));
            nee_pending(a, p, mul(tp, c), ld, L.vid, nf, o);
        }
    }
}

// One step of the bounce/shade loop (shade.comp:543-575, 838-908) for path
// p, with the sun next-event estimate in the place of the emissive NEE
// (VE_FRAME_EMISSIVE: emissive_nee instead): `hit` is the result of the ray along `dir` (ignored for a path marked
// F_TERM), tp/direct/indirect the path state after any pending sun term was
// resolved.  Writes the continuing path's state; the queue appends and the
// AccumPass deposit are left to shade_emit.
// `direct_stored`: `direct` equals the path's p_direct slot (the store is
// skipped while it stays so).
template <int MODE>
__device__ __forceinline__ void shade_step(const FrameArgs& a, uint32_t p, uint4 meta, f3 tp, f3 direct,
                                           f3 indirect, f3 dir, uint4 hit, ShadeOut& o,
                                           bool direct_stored = false, uint32_t share = 0u) {
    constexpr bool EM = (MODE & kModeEm) != 0;
    constexpr bool LB = (MODE & kModeLb) != 0;
    constexpr bool NRC = (MODE & kModeNrc) != 0;
    const uint32_t vi = meta.z & 0xFFFFu;
    uint32_t b = (meta.z >> 16) & 0xFFu;
    const uint32_t flags = meta.z >> 24;
    uint32_t nf = flags & F_TRAIN;
    uint32_t train_slot = 0xFFFFFFFFu;
    // vi indexes the whole view table; `a.views` starts view_offset entries
    // into it when the caller passed one view (the serving primary pass)
    const DevView& v = a.views[vi - a.view_offset];
    o.dview = vi;  // the queue entries of the path's rays carry it
    if (flags & F_TERM) {
        o.do_dep = true;
    } else {
        if (hit.x != kHit) {  // miss (shade.comp:558-564): constant sky
            indirect = add(indirect, mul(mk(v.sky[0], v.sky[1], v.sky[2]), tp));
            o.do_dep = true;
        } else {
            const DevScene S = a.scenes[v.scene];
            const uint32_t mi = hit.w >> 16;
            const DevMaterial m = a.mats[mi & 127u];
            const f3 albedo = mk(m.albedo_rough.x, m.albedo_rough.y, m.albedo_rough.z);
            const float roughness = m.albedo_rough.w, metallic = m.params.x, spec = m.params.y;
            const bool emissive = m.params.z != 0.0f;
            const f3 N = shading_normal(hit.y, dir, S.ntab, S.n_ntab);
            if (emissive) {  // shade.comp:576-583
                const float k = m.params.w;
                f3 em = mul(mk(albedo.x * k, albedo.y * k, albedo.z * k), tp);
                em = mk(gmin(em.x, 20.0f), gmin(em.y, 20.0f), gmin(em.z, 20.0f));
                if (b == 0u) {
                    direct = add(direct, em);
                    direct_stored = false;
                } else {
                    indirect = add(indirect, em);
                }
                // a light seen by a primary ray joins the registry at the end
                // of the frame (shade.comp:585-613)
                if (EM && (v.flags & VE_FRAME_EMISSIVE) && b == 0u) {
                    const uint32_t hx = hit.z & 0xFFFFu, hy = hit.z >> 16, hz = hit.w & 0xFFFFu;
                    const uint32_t lvid = voxel_key(hx, hy, hz) + 1u;
                    if (em_claim(S.em_claim, lvid)) {
                        const uint32_t k2 = atomicAdd(&S.em_state[1], 1u);
                        if (k2 < (1u << kEmClaimLog2))
                            S.em_stage[k2] = EmLight{albedo.x * k, albedo.y * k, albedo.z * k, lvid, hx, hy, hz, 1u};
                    }
                }
            }
            const f3 hp = mk(float(hit.z & 0xFFFFu), float(hit.z >> 16), float(hit.w & 0xFFFFu));
            const f3 sp = add(add(hp, mk(0.5f, 0.5f, 0.5f)), N);
            const f3 sun = mk(v.sun[0], v.sun[1], v.sun[2]);
            // second path vertex: a training path is recorded here, other
            // paths may end with a cached radiance estimate
            bool ended = false;
            if (NRC && b == 1u && !emissive &&
                (v.flags & (VE_FRAME_LEARNED | VE_FRAME_TERMINATE_HASH | VE_FRAME_TRAIN))) {
                const uint32_t hx = hit.z & 0xFFFFu, hy = hit.z >> 16, hz = hit.w & 0xFFFFu;
                const uint32_t cell = hash32((hx >> 3) | ((hy >> 3) << 10) | ((hz >> 3) << 20));
                if ((v.flags & VE_FRAME_TRAIN) && a.ns &&
                    hash32(p ^ (v.frame_index * 0x9E3779B9u)) < a.train_thresh) {
                    nf |= F_TRAIN;
                    train_slot = atomicAdd(&a.counters[CNT_NRC_S], 1u);  // ~2^16 per frame
                    if (train_slot < a.ns_cap) {
                        nrc::TRec t{};
                        t.t0 = tp.x; t.t1 = tp.y; t.t2 = tp.z;
                        const f3 sum = add(direct, indirect);
                        t.s0 = sum.x; t.s1 = sum.y; t.s2 = sum.z;
                        t.cell = cell;
                        a.nt[train_slot] = t;
                        o.sampled = true;
                    } else {
                        train_slot = 0xFFFFFFFFu;
                    }
                    a.p_aux[p] = train_slot;
                } else if (v.flags & (VE_FRAME_LEARNED | VE_FRAME_TERMINATE_HASH)) {
                    bool mlp = false;
                    if ((v.flags & VE_FRAME_LEARNED) && a.nq) {
                        const float4* cs = a.val + 2u * (cell & a.val_mask);
                        const float4 et = cs[0], ey = cs[1];
                        if (et.w < float(kMinCellSamples)) {
                            mlp = a.nrc_ready != 0u;
                        } else {
                            const float ex = (ey.x - et.x) * (ey.x - et.x) / (et.x * et.x + 0.01f);
                            const float eg = (ey.y - et.y) * (ey.y - et.y) / (et.y * et.y + 0.01f);
                            const float eb = (ey.z - et.z) * (ey.z - et.z) / (et.z * et.z + 0.01f);
                            mlp = ((ex + eg) + eb) / 3.0f <= a.fallback_thr;
                        }
                    }
                    if (mlp) {
                        o.want_q = true;
                        ended = true;
                        a.p_tp[p] = st3(tp);
                        a.p_direct[p] = st3(direct);
                        a.p_indirect[p] = st3(indirect);
                    } else {
                        const Avg r = lookup_avg(S, voxel_key(hx, hy, hz) + 1u);
                        if (r.count >= kHashTermMinCount) {
                            indirect = add(indirect, mul(tp, r.rgb));
                            o.do_dep = true;
                            ended = true;
                            o.hash_term = true;
                        }
                    }
                }
                if (o.sampled || o.want_q) {
                    const float inv_l = 1.0f / float(1u << S.depth);
                    const float2 on = oct_encode(N), ov = oct_encode(mk(-dir.x, -dir.y, -dir.z));
                    nrc::QRec qr;
                    qr.px = (hp.x + 0.5f) * inv_l;
                    qr.py = (hp.y + 0.5f) * inv_l;
                    qr.pz = (hp.z + 0.5f) * inv_l;
                    qr.path = p;
                    qr.nx = on.x;
                    qr.ny = on.y;
                    qr.vx = ov.x;
                    qr.vy = ov.y;
                    if (o.sampled) {
                        a.ns[train_slot] = qr;
                    } else {  // parked in the ended path's ray slots until the warp's query append
                        a.p_ray_o[p] = make_float4(qr.px, qr.py, qr.pz, __uint_as_float(qr.path));
                        a.p_ray_d[p] = make_float4(qr.nx, qr.ny, qr.vx, qr.vy);
                    }
                }
            }
            uint32_t rng = meta.y;
            if (EM && (v.flags & VE_FRAME_EMISSIVE)) {
                if (!ended && !emissive && b < 2u)
                    emissive_nee(a, v, S, p, meta.x, b, hit.z & 0xFFFFu, hit.z >> 16, hit.w & 0xFFFFu, N, sp, dir, tp,
                                 albedo, roughness, metallic, spec, rng, nf, o);
            } else if (!ended && !emissive && b < 2u && dot(N, sun) > 0.0f) {
                const f3 brdf = evaluate_brdf(dir, sun, N, albedo, roughness, metallic, spec);
                f3 c = muls(brdf, v.sun_intensity);
                c = mk(gmin(c.x, 20.0f), gmin(c.y, 20.0f), gmin(c.z, 20.0f));
                // the record's last word is the shadow ray's result; until the
                // trace writes it, it holds the count of later records (the
                // pixel's other samples) that take the same result (share)
                a.p_pend[p] = st3(mul(tp, c), __uint_as_float(share == 0xFFFFFFFFu ? 0u : share));
                if (EM) a.p_sdir[p] = make_float4(sun.x, sun.y, sun.z, __uint_as_float(0xFFFFFFFFu));
                nf |= F_PENDING;
                if (share == 0xFFFFFFFFu) {
                    o.sh_shared = true;
                } else {
                    o.app_sh = true;
                    o.sh_owner = share != 0u;
                }
            }
            bool term = false;
            if (ended) {
                // ended by a cache: deposited now (hash) or after inference (network)
            } else if (b + 1u >= v.bounces + 1u) {
                term = true;
            } else {
                const bool use_ggx = metallic * (1.0f - roughness) > 0.5f;
                f3 sdir, bt;
                if (use_ggx) {
                    const f3 V = mk(-dir.x, -dir.y, -dir.z);
                    const f3 H = sample_ggx_vndf(N, V, roughness, rng);
                    sdir = reflect(dir, H);
                    if (dot(sdir, N) <= 0.0f) {
                        sdir = cosine_direction(N, rng);
                        bt = evaluate_brdf(dir, sdir, N, albedo, roughness, metallic, spec);
                    } else {
                        const f3 F0 = mk(0.04f * (1.0f - metallic) + albedo.x * metallic,
                                         0.04f * (1.0f - metallic) + albedo.y * metallic,
                                         0.04f * (1.0f - metallic) + albedo.z * metallic);
                        bt = ggx_throughput(N, V, sdir, H, roughness, F0);
                    }
                } else {
                    sdir = cosine_direction(N, rng);
                    bt = evaluate_brdf(dir, sdir, N, albedo, roughness, metallic, spec);
                }
                f3 ntp = mul(tp, bt);
                if (b + 1u >= 2u) {  // Russian roulette, RR_START_BOUNCE = 2
                    const float pr = gclamp(gmax(ntp.x, gmax(ntp.y, ntp.z)), 0.05f, 0.95f);
                    const float xi = rand01(rng);
                    if (xi > pr) term = true;
                    else ntp = divs(ntp, pr);
                }
                if (!term) {
                    tp = ntp;
                    dir = sdir;
                    b++;
                    o.app_ext = true;
                }
            }
            if (term) {
                if (nf & F_PENDING) nf |= F_TERM;
                else o.do_dep = true;
            }
            if (o.app_ext || (nf & F_PENDING)) {
                o.app_live = true;
                a.p_ray_o[p] = st3(sp);
                a.p_ray_d[p] = st3(dir);
                a.p_tp[p] = st3(tp);
                // radiance that is +0 is flagged instead of stored; direct
                // radiance already in its slot is not stored again
                if (pos_zero(direct)) nf |= F_DZERO;
                else if (!direct_stored) a.p_direct[p] = st3(direct);
                if (pos_zero(indirect)) nf |= F_IZERO;
                else a.p_indirect[p] = st3(indirect);
                meta.y = rng;
                meta.z = vi | (b << 16) | (nf << 24);
                a.p_meta[p] = meta;
            }
        }
    }
    if (o.do_dep) {
        deposit_value(direct, indirect, o.dr, o.dg, o.db, o.dl2);
        const float pr = o.dr, pg = o.dg, pb = o.db;  // the path's value (debug output)
        if (LB) {  // the two channels apart (packRgbL2 of each, shade.comp:162-167)
            float z;
            deposit_value(direct, mk(0.0f, 0.0f, 0.0f), o.dr, o.dg, o.db, z);
            deposit_value(mk(0.0f, 0.0f, 0.0f), indirect, o.ir, o.ig, o.ib, z);
        }
        if (NRC && ((flags | nf) & F_TRAIN)) {  // training path: its target
            const uint32_t k = (nf & F_TRAIN) && !(flags & F_TRAIN) ? train_slot : a.p_aux[p];
            if (k < a.ns_cap) {
                nrc::TRec* t = a.nt + k;
                write_target(t, add(direct, indirect), mk(t->s0, t->s1, t->s2), mk(t->t0, t->t1, t->t2));
            }
        }
        o.dvid = meta.x;
        o.dscene = v.scene;
        o.dview = vi;
        if (a.path_rgb && (v.flags & VE_FRAME_PATH_RGB)) {
            a.path_rgb[3ull * p + 0] = pr;
            a.path_rgb[3ull * p + 1] = pg;
            a.path_rgb[3ull * p + 2] = pb;
        }
    }
}

// The warp-collective part of a shading step: queue appends (live paths,
// extension and shadow rays, learned-cache queries and samples) and the
// warp-aggregated deposit.  Called by all 32 lanes.
template <int MODE>
__device__ __forceinline__ void shade_emit(const FrameArgs& a, uint32_t p, const ShadeOut& o, uint32_t* live_out,
                                           uint32_t* live_cnt, uint32_t* ray_cnt, DepSlot* dep, BlockQ& q,
                                           EmitCounts& cnt) {
    constexpr bool EM = (MODE & kModeEm) != 0;
    constexpr bool LB = (MODE & kModeLb) != 0;
    constexpr bool NRC = (MODE & kModeNrc) != 0;
    const uint3 s = block_append3(o.app_live, o.app_ext, o.app_sh, live_cnt, ray_cnt,
                                  ray_cnt + (CNT_RAYSH - CNT_RAY), q);
    if (o.app_live) live_out[s.x] = p;
    if (o.app_ext) a.rayq[s.y] = make_uint2(p, o.dview);
    if (o.app_sh) a.rayq_sh[s.z] = make_uint2(p | (o.sh_owner ? 0xC0000000u : 0x80000000u), o.dview);
    cnt.ext += o.app_ext ? 1u : 0u;
    cnt.sh += (o.app_sh || o.sh_shared) ? 1u : 0u;
    cnt.shared += o.sh_shared ? 1u : 0u;
    if (NRC && (a.nq || a.ns)) {
        // learned cache: query records move from the path's ray slots into
        // the query queue (capacity = paths, never full)
        const uint32_t kq = warp_append(o.want_q, &a.counters[CNT_NRC_Q]);
        if (o.want_q && kq < a.nq_cap) {
            const float4 r0 = a.p_ray_o[p], r1 = a.p_ray_d[p];
            nrc::QRec q;
            q.px = r0.x; q.py = r0.y; q.pz = r0.z; q.path = __float_as_uint(r0.w);
            q.nx = r1.x; q.ny = r1.y; q.vx = r1.z; q.vy = r1.w;
            a.nq[kq] = q;
        }
        warp_add_stat(&a.stats[ST_NRC_QUERIES], o.want_q ? 1u : 0u);
        warp_add_stat(&a.stats[ST_NRC_SAMPLES], o.sampled ? 1u : 0u);
    }
    if (NRC) warp_add_stat(&a.stats[ST_NRC_HASH], o.hash_term ? 1u : 0u);
    if (EM) {
        const uint32_t kr = warp_append(o.app_res, &a.counters[CNT_RES]);
        if (o.app_res) a.res_list[kr] = p;
        warp_add_stat(&a.stats[ST_EM_NEE], o.em_nee ? 1u : 0u);
    }
    if (LB) {  // recorded at the path's slot; applied per lBuffer row at the end of the frame
        if (o.do_dep) {
            LbRec r;
            r.vid = o.dvid;
            r.slot = p;
            r.d[0] = o.dr; r.d[1] = o.dg; r.d[2] = o.db;
            r.e[0] = o.ir; r.e[1] = o.ig; r.e[2] = o.ib;
            a.lb_rec[p] = r;
            a.lb_key[p] = lb_row(o.dvid);
            cnt.dep++;
        }
    } else {
        warp_deposit(o.do_dep, o.dscene, o.dvid, o.dr, o.dg, o.db, o.dl2, dep, a.scenes, cnt.dep, cnt.drop);
    }
    if (a.remaining) {  // serving: count finished paths per view slot
        const unsigned dm = __ballot_sync(0xffffffffu, o.do_dep);
        if (o.do_dep) {
            const unsigned peers = __match_any_sync(dm, o.dview);
            if (int(lane_id()) == __ffs(peers) - 1) atomicSub(&a.remaining[o.dview], uint32_t(__popc(peers)));
        }
    }
}

// RayPass primary (generate_primary.comp:38-85) + path seeding (emit.comp:39-101).
// FUSED: each seeded path also takes its first shading step here, from the
// hit in registers (the same shade_step the shade pass runs), appending its
// rays and live entry for trace pass 0 / shade pass 1 — the frame's largest
// shade pass never round-trips the path state through memory.
// 4 CTAs/SM (64 registers, ~110 B of spills in the plain instance): the
// kernel is latency-bound, and the extra warps beat the spills (0.49 -> 0.44
// ms per 1080p depth-10 frame).
template <bool COUNT, bool FUSED, int MODE = 0>
__global__ void __launch_bounds__(256, 4) k_primary(FrameArgs a) {
    __shared__ DepSlot dep[FUSED ? 256 : 1];
    const uint32_t tile = blockIdx.x + a.tile_offset;
    const uint32_t vi = find_view(a.views, a.n_views, tile);
    const DevView& v = a.views[vi];
    uint32_t px, py;
    tile_pixel(tile - v.tile_base, v.tiles_x, &px, &py);
    const bool inside = px < v.W && py >= v.g_lo && py < v.g_hi;
    const bool band = py >= v.row_lo && py < v.row_hi;
    const DevScene S = a.scenes[v.scene];
    Hit h;
    h.status = kEscaped;
    h.checks = 0;
    f3 dir = mk(0.0f, 0.0f, 0.0f);
    RayCount rc;
    uint32_t vid = 0, word = 0;
    if (inside) {
        const float ndx = (float(px) + 0.5f) / float(v.W) * 2.0f - 1.0f;
        const float ndy = (float(py) + 0.5f) / float(v.H) * 2.0f - 1.0f;
        const f3 plane = mk(v.cam[4], v.cam[5], v.cam[6]);
        const f3 right = mk(v.cam[8], v.cam[9], v.cam[10]);
        const f3 up = mk(v.cam[12], v.cam[13], v.cam[14]);
        dir = normalize(sub(add(plane, muls(right, ndx)), muls(up, ndy)));
        h = raycast<COUNT>(S.nodes, S.n_words, S.depth, S.top, S.top_level, mk(v.cam[0], v.cam[1], v.cam[2]), dir,
                           v.cc_primary, rc);
        if (h.status == kHit) {
            vid = voxel_key(h.x, h.y, h.z) + 1u;
            word = __ldg(S.nodes + h.id);  // the hit leaf's word, for shading
        }
        const uint32_t pix = py * v.W + px;
        a.gbuf[v.pix_base + pix] = make_uint4(h.checks, h.status == kHit ? h.material : 0u,
                                              h.status == kHit ? h.id : 0u, vid);
        if (v.flags & VE_FRAME_SCHEDULED)  // paths come from the shade list: keep the hit
            a.hitinfo[v.pix_base + pix] = make_uint4(word, h.x | (h.y << 16), h.z | (h.material << 16), 0u);
    }
    const bool spawn = inside && band && vid != 0u && !(v.flags & VE_FRAME_SCHEDULED);
    if (FUSED && !(v.flags & VE_FRAME_SCHEDULED)) {
        // the warp's (pixel, sample) pairs in chunks of 32, pixel-major: the
        // lanes of one chunk hold consecutive path slots (a row of the warp's
        // 8 x 4 pixel block), so path-state stores and queue entries stay
        // coalesced.  Lane i traced pixel i of the block.
        __shared__ BlockQ bq[2];
        EmitCounts cnt;
        const uint32_t lane = lane_id();
        const uint32_t spp = v.spp;  // one view per block: uniform
        const uint32_t pix = py * v.W + px;
        const uint32_t hxy = h.x | (h.y << 16), hzm = h.z | (h.material << 16);
        for (uint32_t it = 0; it < spp; it++) {
            const uint32_t qi = it * 32u + lane;
            const uint32_t src = qi / spp, s = qi - src * spp;
            const bool sp = __shfl_sync(0xffffffffu, spawn ? 1 : 0, int(src)) != 0;
            const uint32_t svid = __shfl_sync(0xffffffffu, vid, int(src));
            const uint32_t spix = __shfl_sync(0xffffffffu, pix, int(src));
            const uint32_t sword = __shfl_sync(0xffffffffu, word, int(src));
            const uint32_t sxy = __shfl_sync(0xffffffffu, hxy, int(src));
            const uint32_t szm = __shfl_sync(0xffffffffu, hzm, int(src));
            const f3 sdir = mk(__shfl_sync(0xffffffffu, dir.x, int(src)), __shfl_sync(0xffffffffu, dir.y, int(src)),
                               __shfl_sync(0xffffffffu, dir.z, int(src)));
            const uint32_t p = uint32_t(v.path_base + (unsigned long long)spix * spp + s);
            ShadeOut o;
            if (sp) {
                const uint32_t list_idx = spix * spp + s;
                // emit.comp:171-174
                const uint32_t sample_idx = v.frame_index + spix * 2654435761u + list_idx * 1442695040u;
                const uint32_t rng = (sample_idx << 8) & 0xFFFFFF00u;
                // the samples of a pixel start at the same hit with the same
                // direction: one sun shadow ray (sample 0's) serves them all
                // (share: sample 0 carries the count of the others, each of
                // which casts none).  Emissive batches keep their own.
                const uint32_t share = (!(MODE & kModeEm) && spp > 1u) ? (s == 0u ? spp - 1u : 0xFFFFFFFFu) : 0u;
                shade_step<MODE>(a, p, make_uint4(svid, rng, vi + a.view_offset, spix), mk(1.0f, 1.0f, 1.0f),
                           mk(0.0f, 0.0f, 0.0f), mk(0.0f, 0.0f, 0.0f), sdir, make_uint4(kHit, sword, sxy, szm), o,
                           false, share);
            }
            shade_emit<MODE>(a, p, o, a.live[1], &a.counters[CNT_LIVE + 1], &a.counters[CNT_RAY + 0],
                           dep + (threadIdx.x & ~31u), bq[it & 1u], cnt);
        }
        flush_counts(cnt, a.stats);
    }
    const uint32_t q = FUSED ? 0u : warp_append(spawn, &a.counters[CNT_LIVE + 0], v.spp);
    if (!FUSED && spawn) {
        const uint32_t pix = py * v.W + px;
        for (uint32_t s = 0; s < v.spp; s++) {
            const uint32_t p = uint32_t(v.path_base + (unsigned long long)pix * v.spp + s);
            const uint32_t list_idx = pix * v.spp + s;
            // emit.comp:171-174
            const uint32_t sample_idx = v.frame_index + pix * 2654435761u + list_idx * 1442695040u;
            const uint32_t rng = (sample_idx << 8) & 0xFFFFFF00u;
            a.p_ray_d[p] = st3(dir);
            a.p_tp[p] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
            a.p_hit[p] = make_uint4(kHit, word, h.x | (h.y << 16), h.z | (h.material << 16));
            a.p_meta[p] = make_uint4(vid, rng, (vi + a.view_offset) | ((F_DZERO | F_IZERO) << 24), pix);
            a.live[0][q + s] = uint32_t(p);
        }
    }
    warp_add_stat(&a.stats[ST_RAYS_PRIMARY], inside && band ? 1u : 0u);
    warp_add_stat(&a.stats[ST_PATHS], spawn ? v.spp : 0u);
    if (a.remaining) {  // the whole block belongs to one view
        uint32_t sp = spawn ? v.spp : 0u;
        for (int o = 16; o > 0; o >>= 1) sp += __shfl_xor_sync(0xffffffffu, sp, o);
        if (lane_id() == 0 && sp) atomicAdd(&a.remaining[vi + a.view_offset], sp);
    }
    if (COUNT) {
        warp_add_stat(&a.stats[ST_FETCH], rc.fetch);
        warp_add_stat(&a.stats[ST_STEPS], rc.steps);
    }
}

// Latency-bound on the path-state loads: more resident warps win as long as
// the spills stay small.  The plain instance runs 5 CTAs/SM (48 registers,
// 0.414 -> 0.397 ms per 1080p depth-10 frame against 4); the emissive,
// lBuffer and learned instances keep 4 (at 5 they would spill 190-340 B).
// Each instance's grid is sized from its own occupancy (shade_grid), so none
// runs part of its grid as a second wave.
constexpr int shade_ctas(int mode) { return mode == 0 ? 5 : 4; }
template <int MODE = 0>
__global__ void __launch_bounds__(256, shade_ctas(MODE)) k_shade(FrameArgs a, uint32_t pass) {
    constexpr bool EM = (MODE & kModeEm) != 0;
    __shared__ DepSlot dep[256];
    const uint32_t n = a.counters[CNT_LIVE + pass];
    const uint32_t* live_in = a.live[pass & 1u];
    uint32_t* live_out = a.live[(pass + 1u) & 1u];
    uint32_t* live_cnt = &a.counters[CNT_LIVE + pass + 1u];
    uint32_t* ray_cnt = &a.counters[CNT_RAY + pass];
    __shared__ BlockQ bq[2];
    EmitCounts cnt;
    uint32_t it = 0;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x, it++) {
        const uint32_t i = base + threadIdx.x;
        const bool valid = i < n;
        const uint32_t p = valid ? live_in[i] : 0u;
        ShadeOut o;
        if (valid) {
            const uint4 meta = a.p_meta[p];
            const float4 pe = a.p_pend[p];  // read with the rest: no load waits on the flags
            const uint32_t want = EM ? __float_as_uint(a.p_sdir[p].w) : 0xFFFFFFFFu;
            const uint32_t flags = meta.z >> 24;
            // issued with the rest and discarded when flagged: no load waits on the flags
            const float4 d4 = a.p_direct[p], i4 = a.p_indirect[p];
            f3 direct = (flags & F_DZERO) ? mk(0.0f, 0.0f, 0.0f) : ld3(d4);
            f3 indirect = (flags & F_IZERO) ? mk(0.0f, 0.0f, 0.0f) : ld3(i4);
            bool direct_stored = !(flags & F_DZERO);
            if ((flags & F_PENDING) && __float_as_uint(pe.w) == want) {
                // the sun term belongs to the bounce that cast the shadow ray:
                // the stored one when the path ended there, else the one before
                const uint32_t b = (meta.z >> 16) & 0xFFu;
                if (((flags & F_TERM) ? b : b - 1u) == 0u) {
                    direct = add(direct, ld3(pe));
                    direct_stored = false;
                } else {
                    indirect = add(indirect, ld3(pe));
                }
            }
            const uint4 hit = (flags & F_TERM) ? make_uint4(0u, 0u, 0u, 0u) : a.p_hit[p];
            shade_step<MODE>(a, p, meta, ld3(a.p_tp[p]), direct, indirect, ld3(a.p_ray_d[p]), hit, o,
                             direct_stored);
        }
        shade_emit<MODE>(a, p, o, live_out, live_cnt, ray_cnt, dep + (threadIdx.x & ~31u), bq[it & 1u], cnt);
    }
    flush_counts(cnt, a.stats);
}

// ---------------------------------------------------------------------------
// Importance-aware voxel scheduling (schedule.comp, rank.comp, threshold.comp,
// emit.comp), one view per frame.  Differences from the reference, for
// determinism: a voxel's representative pixel is its smallest pixel index
// (the reference keeps the first pixel to claim it, in a scrambled
// workgroup order), the shade list is ordered by representative pixel
// starting at a per-frame rotation of the pixel index (a prefix sum instead
// of atomic appends; the rotation spreads the shading budget's cut over the
// image from frame to frame), and paths start from the stored primary hit
// instead of re-casting the primary ray.
__device__ __forceinline__ uint32_t sched_rotation(uint32_t frame, uint32_t npix) {
    return uint32_t((unsigned long long)(frame * 0x9E3779B9u) % npix);
}
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t claim_hash(uint32_t vid) {  // schedule.comp claimHash
    uint32_t x = vid;
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    return x;
}

// schedule.comp: claim the voxel of every hit pixel, count its pixels and
// keep its smallest pixel index.
__global__ void __launch_bounds__(256) k_sched_claim(FrameArgs a) {
    const DevView& v = a.views[0];
    const uint32_t npix = v.W * v.H;
    for (uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x; pix < npix; pix += gridDim.x * blockDim.x) {
        const uint32_t vid = a.gbuf[v.pix_base + pix].w;
        if (vid == 0u) continue;
        uint32_t h = claim_hash(vid) & a.claim_mask;
        for (uint32_t q = 0; q < kClaimProbes; q++, h = (h + 1u) & a.claim_mask) {
            const uint32_t prev = atomicCAS(&a.claim_key[h], 0u, vid);
            if (prev == 0u || prev == vid) {
                atomicMin(&a.claim_pix[h], pix);
                atomicAdd(&a.claim_cnt[h], 1u);
                break;
            }
        }
    }
}

__device__ __forceinline__ int claim_find(const FrameArgs& a, uint32_t vid) {
    uint32_t h = claim_hash(vid) & a.claim_mask;
    for (uint32_t q = 0; q < kClaimProbes; q++, h = (h + 1u) & a.claim_mask) {
        const uint32_t k = a.claim_key[h];
        if (k == vid) return int(h);
        if (k == 0u) return -1;
    }
    return -1;
}

// rank.comp: importance = w_pix * coverage + w_var * variance (the voxel's
// radiance-cache variance from the previous frames, on the VARIANCE view's
// scale), tiers from the previous frame's thresholds, histogram for the
// next ones.  sched_n[j] = paths of the voxel whose representative pixel
// is pix, j = (pix - rotation) mod pixels.
__global__ void __launch_bounds__(256) k_sched_rank(FrameArgs a) {
    const DevView& v = a.views[0];
    const DevScene S = a.scenes[v.scene];
    const uint32_t npix = v.W * v.H;
    const float t_high = a.rank[0], t_mid = a.rank[1];
    const uint32_t rot = sched_rotation(v.frame_index, npix);
    uint32_t* hist = reinterpret_cast<uint32_t*>(a.rank + 2);
    uint32_t nvox = 0;
    for (uint32_t base = blockIdx.x * blockDim.x; base < npix; base += gridDim.x * blockDim.x) {
        const uint32_t pix = base + threadIdx.x;
        uint32_t n = 0;
        if (pix < npix) {
            const uint32_t vid = a.gbuf[v.pix_base + pix].w;
            const int c = vid ? claim_find(a, vid) : -1;
            if (c >= 0 && a.claim_pix[c] == pix) {
                nvox++;
                const float pn = gclamp(float(a.claim_cnt[c]) / gmax(v.pix_norm, 1.0f), 0.0f, 1.0f);
                float vn;
                if ((v.flags & VE_FRAME_LBUFFER) && S.lbuf) {  // rank.comp:107 on the lBuffer's own scale
                    vn = gclamp(lb_indirect_variance(S.lbuf, vid) / gmax(v.variance_norm, 1.0f), 0.0f, 1.0f);
                } else {
                    const Avg av = lookup_avg(S, vid);
                    const float var = av.count >= 2u ? av.var : 0.0f;
                    vn = gclamp(var * (255.0f * 255.0f) / gmax(v.variance_norm, 1.0f), 0.0f, 1.0f);
                }
                const float imp = v.w_pix * pn + v.w_var * vn;
                n = imp >= t_high ? 2u : (imp >= t_mid ? 1u : v.min_samples);
                uint32_t bin = uint32_t(imp * float(kRankBins));
                if (bin >= kRankBins) bin = kRankBins - 1u;
                atomicAdd(&hist[bin], 1u);
            }
            a.sched_n[pix >= rot ? pix - rot : pix + (npix - rot)] = n;
        }
    }
    warp_add_stat(&a.stats[ST_SCHED_VOXELS], nvox);
}

// The shade list: n entries {vid, pixel} at the rotated pixel's prefix-sum
// offset, cut at the shading budget; the last position publishes the entry
// count.
__global__ void __launch_bounds__(256) k_sched_list(FrameArgs a) {
    const DevView& v = a.views[0];
    const uint32_t npix = v.W * v.H;
    const uint32_t cap = min(a.shade_cap, v.budget);
    const uint32_t rot = sched_rotation(v.frame_index, npix);
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < npix; j += gridDim.x * blockDim.x) {
        const uint32_t n = a.sched_n[j], off = a.sched_off[j];
        if (j + 1u == npix) a.counters[CNT_SCHED] = min(off + n, cap);
        const uint32_t pix = j < npix - rot ? j + rot : j - (npix - rot);
        if (n == 0u) continue;
        const uint32_t vid = a.gbuf[v.pix_base + pix].w;
        for (uint32_t e = 0; e < n && off + e < cap; e++) a.shade_list[off + e] = make_uint2(vid, pix);
    }
}

// threshold.comp: the next frame's thresholds from this frame's histogram
// (top_frac of the voxels above t_high, the next mid_frac above t_mid).
__global__ void k_sched_threshold(float* rank, const DevView* views) {
    uint32_t* hist = reinterpret_cast<uint32_t*>(rank + 2);
    uint32_t total = 0;
    for (uint32_t b = 0; b < kRankBins; b++) total += hist[b];
    if (total == 0u) {
        rank[0] = __int_as_float(0x7f800000);   // +inf
        rank[1] = __int_as_float(0xff800000);   // -inf
        return;
    }
    const float top = gclamp(views[0].top_frac, 0.0f, 1.0f);
    const float mid = gclamp(views[0].mid_frac, 0.0f, 1.0f - top);
    const uint32_t top_n = uint32_t(top * float(total)), topmid_n = uint32_t((top + mid) * float(total));
    uint32_t cum = 0, hb = kRankBins, mb = kRankBins;
    for (int b = int(kRankBins) - 1; b >= 0; b--) {
        cum += hist[b];
        if (hb == kRankBins && cum >= top_n) hb = uint32_t(b);
        if (mb == kRankBins && cum >= topmid_n) mb = uint32_t(b);
        if (hb != kRankBins && mb != kRankBins) break;
    }
    if (hb == kRankBins) hb = kRankBins - 1u;
    if (mb == kRankBins) mb = kRankBins - 1u;
    rank[0] = float(hb) / float(kRankBins);
    rank[1] = float(mb) / float(kRankBins);
}

// emit.comp: one path per shade-list entry, from the representative pixel's
// primary hit, list index i seeding the RNG; its first shading step runs
// here as in the fused primary pass.
template <int MODE = 0>
__global__ void __launch_bounds__(256, 4) k_sched_emit(FrameArgs a) {
    __shared__ DepSlot dep[256];
    const DevView& v = a.views[0];
    const uint32_t n = a.counters[CNT_SCHED];
    const f3 plane = mk(v.cam[4], v.cam[5], v.cam[6]);
    const f3 right = mk(v.cam[8], v.cam[9], v.cam[10]);
    const f3 up = mk(v.cam[12], v.cam[13], v.cam[14]);
    __shared__ BlockQ bq[2];
    EmitCounts cnt;
    uint32_t n_paths = 0, it = 0;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x, it++) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t p = uint32_t(v.path_base) + i;
        ShadeOut o;
        if (i < n) {
            const uint2 e = a.shade_list[i];
            const uint32_t pix = e.y, px = pix % v.W, py = pix / v.W;
            const float ndx = (float(px) + 0.5f) / float(v.W) * 2.0f - 1.0f;
            const float ndy = (float(py) + 0.5f) / float(v.H) * 2.0f - 1.0f;
            const f3 dir = normalize(sub(add(plane, muls(right, ndx)), muls(up, ndy)));
            const uint4 hi = a.hitinfo[v.pix_base + pix];
            // emit.comp:171-174 with listIdx = the shade-list index
            const uint32_t sample_idx = v.frame_index + pix * 2654435761u + i * 1442695040u;
            const uint32_t rng = (sample_idx << 8) & 0xFFFFFF00u;
            shade_step<MODE>(a, p, make_uint4(e.x, rng, 0u + a.view_offset, pix), mk(1.0f, 1.0f, 1.0f), mk(0.0f, 0.0f, 0.0f),
                       mk(0.0f, 0.0f, 0.0f), dir, make_uint4(kHit, hi.x, hi.y, hi.z), o);
            n_paths++;
        }
        shade_emit<MODE>(a, p, o, a.live[1], &a.counters[CNT_LIVE + 1], &a.counters[CNT_RAY + 0], dep + (threadIdx.x & ~31u),
                       bq[it & 1u], cnt);
    }
    flush_counts(cnt, a.stats);
    warp_add_stat(&a.stats[ST_PATHS], n_paths);
    warp_add_stat(&a.stats[ST_SCHED_PATHS], n_paths);
}

// ---------------------------------------------------------------------------
// End-of-frame commits of emissive frames.
// ---------------------------------------------------------------------------
// Registry: sort keys = the staged lights' vids (unused slots ~0), values =
// staging indices.
__global__ void __launch_bounds__(256) k_em_keys(const DevScene* scenes, uint32_t sc, uint32_t* keys, uint32_t* vals) {
    const DevScene S = scenes[sc];
    constexpr uint32_t cap = 1u << kEmClaimLog2;
    const uint32_t n = min(S.em_state[1], cap);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cap; i += gridDim.x * blockDim.x) {
        keys[i] = i < n ? S.em_stage[i].vid : 0xFFFFFFFFu;
        vals[i] = i;
    }
}
// ... the staged lights in vid order fill the registry's free records (one
// block: every thread reads the counts before thread 0 updates them).
__global__ void __launch_bounds__(1024) k_em_append(const DevScene* scenes, uint32_t sc, const uint32_t* order,
                                                    unsigned long long* stats) {
    const DevScene S = scenes[sc];
    const uint32_t count = min(S.em_state[0], kEmCapacity);
    const uint32_t n = min(S.em_state[1], 1u << kEmClaimLog2);
    const uint32_t add = min(n, kEmCapacity - count);
    for (uint32_t i = threadIdx.x; i < add; i += blockDim.x) S.em_list[count + i] = S.em_stage[order[i]];
    __syncthreads();
    if (threadIdx.x == 0) {
        S.em_state[0] = count + add;
        S.em_state[1] = 0u;
        atomicAdd(&stats[ST_EM_LIGHTS], (unsigned long long)(count + add));
    }
}
// Reservoirs: each voxel keeps the reservoir of its winning path (the
// largest slot among the frame's bounce-0 paths on it).
__global__ void __launch_bounds__(256) k_res_commit(FrameArgs a) {
    const uint32_t n = a.counters[CNT_RES];
    uint32_t w = 0;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        if (i < n) {
            const uint32_t p = a.res_list[i];
            const PathRes pr = a.p_res[p];
            ResEntry* t = a.scenes[pr.scene].res + pr.entry;
            if (t->winner == p + 1u) {
                t->light_idx = pr.r.light_idx;
                t->light_vid = pr.r.light_vid;
                t->seed = pr.r.seed;
                t->wsum = pr.r.wsum;
                t->m = pr.r.m;
                t->target = pr.r.target;
                t->winner = 0u;
                w++;
            }
        }
    }
    warp_add_stat(&a.stats[ST_RES_WRITES], w);
}

// ---------------------------------------------------------------------------
// End-of-frame AccumPass of lBuffer frames.  Deposits sit at their path
// slots, so a stable radix sort of their rows (15 bits) orders them by
// (row, path slot); each row's run is then applied by one warp, lane i
// holding slot i of the row in registers: the reference's sequential slot
// scan becomes one ballot per deposit.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_lb_bounds(const uint32_t* keys, uint32_t n, uint32_t* start,
                                                   uint32_t* end) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t row = keys[i];
        if (row == 0u) continue;  // paths without a deposit
        if (i == 0u || keys[i - 1] != row) start[row] = i;
        if (i + 1u == n || keys[i + 1] != row) end[row] = i + 1u;
    }
}
__global__ void __launch_bounds__(256) k_lb_apply(const DevScene* scenes, const DevView* views, const LbRec* rec,
                                                  const uint32_t* order, const uint32_t* start,
                                                  const uint32_t* end) {
    const DevView& v = views[0];
    uint32_t* lb = scenes[v.scene].lbuf;
    const LbParams P = v.lb;
    const uint32_t lane = lane_id();
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < kLbWidth; r += warps) {
        const uint32_t b = start[r], e = end[r];
        if (b == e) continue;
        uint32_t* gs = lb + size_t(r) * kLbRowWords + lane * kLbStride;
        uint32_t s[kLbStride];
#pragma unroll
        for (int k = 0; k < int(kLbStride); k++) s[k] = gs[k];
        for (uint32_t i0 = b; i0 < e; i0 += 32u) {
            // the next 32 deposits fetched by the 32 lanes at once, then
            // applied one by one from shuffles
            LbRec mine{};
            if (i0 + lane < e) mine = rec[order[i0 + lane]];
            const uint32_t cnt = min(32u, e - i0);
            for (uint32_t k = 0; k < cnt; k++) {
                LbRec x;
                x.vid = __shfl_sync(0xffffffffu, mine.vid, int(k));
#pragma unroll
                for (int q = 0; q < 3; q++) {
                    x.d[q] = __shfl_sync(0xffffffffu, mine.d[q], int(k));
                    x.e[q] = __shfl_sync(0xffffffffu, mine.e[q], int(k));
                }
                uint32_t d[4], c[4];
                lb_pack(x.d, d);
                lb_pack(x.e, c);
                // the scan's stop: the vid's slot or the first empty one
                // (empty slots only follow the used ones: none is ever cleared)
                const unsigned m = __ballot_sync(0xffffffffu, s[0] == x.vid || s[0] == 0u);
                if (m) {
                    if (int(lane) == __ffs(m) - 1) {
                        if (s[0] == 0u) s[0] = x.vid;
                        lb_update(s, x.vid, d, c, P);
                    }
                } else {  // no slot: the least recently used one (first of equal times)
                    uint32_t t = s[11], who = lane;
                    for (int o = 16; o > 0; o >>= 1) {
                        const uint32_t t2 = __shfl_xor_sync(0xffffffffu, t, o);
                        const uint32_t w2 = __shfl_xor_sync(0xffffffffu, who, o);
                        if (t2 < t || (t2 == t && w2 < who)) {
                            t = t2;
                            who = w2;
                        }
                    }
                    if (t != 0xFFFFFFFFu && lane == who) lb_reset(s, x.vid, d, c, P.time);
                }
            }
        }
#pragma unroll
        for (int k = 0; k < int(kLbStride); k++) gs[k] = s[k];
    }
}

__global__ void __launch_bounds__(256) k_iota(uint32_t* v, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] = i;
}

// Launches of the shading kernels' instances for a mode (kModeEm | kModeLb,
// or kModeNrc alone: the API refuses cache-terminated paths with the others).
template <bool COUNT>
static void launch_primary(int mode, uint32_t grid, cudaStream_t st, const FrameArgs& a) {
    switch (mode & ~kModeNrc) {
        case 0: k_primary<COUNT, true, 0><<<grid, 256, 0, st>>>(a); break;
        case kModeEm: k_primary<COUNT, true, kModeEm><<<grid, 256, 0, st>>>(a); break;
        case kModeLb: k_primary<COUNT, true, kModeLb><<<grid, 256, 0, st>>>(a); break;
        default: k_primary<COUNT, true, kModeEm | kModeLb><<<grid, 256, 0, st>>>(a); break;
    }
}
static void launch_shade(int mode, uint32_t grid, cudaStream_t st, const FrameArgs& a, uint32_t pass) {
    switch (mode) {
        case 0: k_shade<0><<<grid, 256, 0, st>>>(a, pass); break;
        case kModeEm: k_shade<kModeEm><<<grid, 256, 0, st>>>(a, pass); break;
        case kModeLb: k_shade<kModeLb><<<grid, 256, 0, st>>>(a, pass); break;
        case kModeNrc: k_shade<kModeNrc><<<grid, 256, 0, st>>>(a, pass); break;
        default: k_shade<kModeEm | kModeLb><<<grid, 256, 0, st>>>(a, pass); break;
    }
}
static void launch_sched_emit(int mode, uint32_t grid, cudaStream_t st, const FrameArgs& a) {
    switch (mode & ~kModeNrc) {
        case 0: k_sched_emit<0><<<grid, 256, 0, st>>>(a); break;
        case kModeEm: k_sched_emit<kModeEm><<<grid, 256, 0, st>>>(a); break;
        case kModeLb: k_sched_emit<kModeLb><<<grid, 256, 0, st>>>(a); break;
        default: k_sched_emit<kModeEm | kModeLb><<<grid, 256, 0, st>>>(a); break;
    }
}

// Staging of a learned-cache query in a frame (runs in the encode kernel, at
// full occupancy): the path state its deposit needs, gathered from the
// path's random slot into the query's own row.
struct StagePath {
    FrameArgs a;
    __device__ __forceinline__ void operator()(uint32_t row, const nrc::QRec& q) const {
        const uint32_t p = q.path;
        const uint4 meta = a.p_meta[p];
        const DevView& v = a.views[meta.z & 0xFFFFu];
        const float4 tp = a.p_tp[p], di = a.p_direct[p], in = a.p_indirect[p];
        const uint32_t sc = v.scene | ((v.flags & VE_FRAME_PATH_RGB) ? 0x80000000u : 0u);
        a.nstage[3ull * row + 0] = make_float4(tp.x, tp.y, tp.z, __uint_as_float(p));
        a.nstage[3ull * row + 1] = make_float4(di.x, di.y, di.z, __uint_as_float(meta.x));
        a.nstage[3ull * row + 2] = make_float4(in.x, in.y, in.z, __uint_as_float(sc));
    }
};

// Epilogue of the learned cache's inference in a frame: the query's path
// gets throughput x prediction (negative channels read as zero) added to its
// indirect radiance and is deposited like any finished path.  Runs inside
// k_nrc_infer, on the 128 threads of a warpgroup (warp-aggregated deposits
// through the group's free operand tile).
struct ApplyDeposit {
    FrameArgs a;
    __device__ __forceinline__ void operator()(uint8_t* scratch, uint32_t row, bool valid, const float (&y)[3]) const {
        float dr = 0.0f, dg = 0.0f, db = 0.0f, dl2 = 0.0f;
        uint32_t dvid = 0, dscene = 0;
        if (valid) {
            const float4 s0 = a.nstage[3ull * row + 0], s1 = a.nstage[3ull * row + 1], s2 = a.nstage[3ull * row + 2];
            const f3 pred = mk(y[0] > 0.0f ? y[0] : 0.0f, y[1] > 0.0f ? y[1] : 0.0f, y[2] > 0.0f ? y[2] : 0.0f);
            const f3 tp = ld3(s0);
            const f3 indirect = add(ld3(s2), mul(tp, pred));
            deposit_value(ld3(s1), indirect, dr, dg, db, dl2);
            dvid = __float_as_uint(s1.w);
            const uint32_t sc = __float_as_uint(s2.w);
            dscene = sc & 0x7FFFFFFFu;
            if (a.path_rgb && (sc & 0x80000000u)) {
                const uint32_t p = __float_as_uint(s0.w);
                a.path_rgb[3ull * p + 0] = dr;
                a.path_rgb[3ull * p + 1] = dg;
                a.path_rgb[3ull * p + 2] = db;
            }
        }
        DepSlot* dep = reinterpret_cast<DepSlot*>(scratch) + (threadIdx.x & 96u);
        uint32_t n_dep = 0, n_drop = 0;
        warp_deposit(valid, dscene, dvid, dr, dg, db, dl2, dep, a.scenes, n_dep, n_drop);
        warp_add_stat(&a.stats[ST_DEPOSITS], n_dep);
        warp_add_stat(&a.stats[ST_DROPPED], n_drop);
    }
};

__device__ __forceinline__ float aces(float x) {  // final.frag:11-18
    const float v = (x * (2.51f * x + 0.03f)) / (x * (2.43f * x + 0.59f) + 0.14f);
    return gclamp(v, 0.0f, 1.0f);
}

// AvgPass (resolve.comp:362-382 with resolveDefault :224-261,
// reconstructTimeout :193-219 and the visualisation modes) + tonemap.
// LB: the batch has VE_FRAME_LBUFFER views.
template <bool LB = false>
__global__ void __launch_bounds__(256) k_resolve(FrameArgs a) {
    const uint32_t tile = blockIdx.x;
    const uint32_t vi = find_view(a.views, a.n_views, tile);
    const DevView& v = a.views[vi];
    uint32_t px, py;
    tile_pixel(tile - v.tile_base, v.tiles_x, &px, &py);
    if (px >= v.W || py < v.row_lo || py >= v.row_hi) return;
    const DevScene S = a.scenes[v.scene];
    const uint32_t W = v.W, H = v.H;
    const uint32_t gp = v.pix_base + py * W + px;
    const uint4 g = a.gbuf[gp];
    const uint32_t checks = g.x, mat = g.y, node = g.z, vid = g.w;
    const f3 sky = mk(v.sky[0], v.sky[1], v.sky[2]);
    f3 col = mk(0.0f, 0.0f, 0.0f);
    auto reconstruct = [&]() {
        f3 sum = mk(0.0f, 0.0f, 0.0f);
        float ws = 0.0f;
        const int R = int(v.recon_radius);
        for (int dy = -R; dy <= R; dy++)
            for (int dx = -R; dx <= R; dx++) {
                if (dx == 0 && dy == 0) continue;
                const int qx = int(px) + dx, qy = int(py) + dy;
                if (qx < 0 || qy < 0 || qx >= int(W) || qy >= int(H)) continue;
                const uint4 nd = a.gbuf[v.pix_base + uint32_t(qy) * W + uint32_t(qx)];
                if (nd.w == 0u || nd.x >= v.cc_primary) continue;
                const Avg na = lookup_view<LB>(v, S, nd.w);
                if (na.count == 0u) continue;
                const float dist = float(dx * dx + dy * dy);
                const float w = float(na.count < 32u ? na.count : 32u) / (1.0f + dist * 0.15f);
                sum = add(sum, muls(na.rgb, w));
                ws += w;
            }
        return ws > 0.0001f ? divs(sum, ws) : sky;
    };
    auto miss = [&]() { return checks >= v.cc_primary ? reconstruct() : sky; };
    switch (v.render_type) {
        case VE_RENDER_STRUCTURE: {
            const float s = float(checks) / 65.0f;
            col = mk(s, s, s);
            break;
        }
        case VE_RENDER_ALBEDO:
            if (vid == 0u) col = miss();
            else if (mat != 0u && mat < 127u) {
                const float4 m = a.mats[mat].albedo_rough;
                col = mk(m.x, m.y, m.z);
            }
            break;
        case VE_RENDER_NORMAL:
            if (vid == 0u) col = miss();
            else {
                const uint32_t w = fetch_node(S.nodes, S.n_words, node);
                if ((w >> 31) || (S.ntab && ball_index(w) != 0u)) {
                    const f3 nn = shading_normal(w, mk(0.0f, 0.0f, 1.0f), S.ntab, S.n_ntab);
                    col = mk(nn.x * 0.5f + 0.5f, nn.y * 0.5f + 0.5f, nn.z * 0.5f + 0.5f);
                }
            }
            break;
        case VE_RENDER_VOXELID:
            if (vid == 0u) col = miss();
            else {
                const uint32_t hid = vid - 1u;
                col = mk(float((hid + 1u) % 255u) / 255.0f, float(((hid + 1u) / 255u) % 255u) / 255.0f,
                         float(((hid + 1u) / (255u * 255u)) % 255u) / 255.0f);
            }
            break;
        case VE_RENDER_VARIANCE:
            if (vid == 0u) col = miss();
            else {
                const Avg c = lookup_view<LB>(v, S, vid);
                const float var = c.count >= 2u ? c.var : 0.0f;
                const float sc = gclamp(var * (255.0f * 255.0f) / gmax(v.variance_norm, 1.0f), 0.0f, 1.0f);
                col = mk(sc, sc, sc);
            }
            break;
        default: {
            if (vid == 0u) {
                col = miss();
                break;
            }
            const Avg c = lookup_view<LB>(v, S, vid);
            if (c.count >= 128u && c.var < 0.02f) {
                col = c.rgb;
                break;
            }
            f3 sum = muls(c.rgb, float(c.count));
            float ws = float(c.count);
            const int dxs[4] = {1, -1, 0, 0}, dys[4] = {0, 0, 1, -1};
            for (int k = 0; k < 4; k++) {
                const int qx = int(px) + dxs[k], qy = int(py) + dys[k];
                if (qx < 0 || qy < 0 || qx >= int(W) || qy >= int(H)) continue;
                const uint32_t nv = a.gbuf[v.pix_base + uint32_t(qy) * W + uint32_t(qx)].w;
                if (nv == 0u || nv == vid) continue;
                const Avg na = lookup_view<LB>(v, S, nv);
                if (na.count == 0u) continue;
                const f3 dd = sub(na.rgb, c.rgb);
                const float dc = sqrtf(dot(dd, dd));
                const float wc = expf(-dc * 6.0f);
                const float wv = 1.0f / (1.0f + na.var * 32.0f);
                const float w = wc * wv * float(na.count < 32u ? na.count : 32u);
                sum = add(sum, muls(na.rgb, w));
                ws += w;
            }
            if (ws > 0.0001f) col = divs(sum, ws);
            break;
        }
    }
    if (a.out_vid) a.out_vid[gp] = vid;
    if (a.out_node) a.out_node[gp] = node;
    if (a.out_rgb) {
        a.out_rgb[3ull * gp + 0] = col.x;
        a.out_rgb[3ull * gp + 1] = col.y;
        a.out_rgb[3ull * gp + 2] = col.z;
    }
    const f3 m = mk(aces(col.x), aces(col.y), aces(col.z));
    if (a.out_mapped) {
        a.out_mapped[3ull * gp + 0] = m.x;
        a.out_mapped[3ull * gp + 1] = m.y;
        a.out_mapped[3ull * gp + 2] = m.z;
    }
    // the framebuffer's unsigned-normalised store of FragColor = (mapped, 1):
    // clamp to [0, 1], scale by 255, round to nearest
    if (a.out_mapped8)
        a.out_mapped8[gp] = make_uchar4(uint8_t(uint32_t(gclamp(m.x, 0.0f, 1.0f) * 255.0f + 0.5f)),
                                        uint8_t(uint32_t(gclamp(m.y, 0.0f, 1.0f) * 255.0f + 0.5f)),
                                        uint8_t(uint32_t(gclamp(m.z, 0.0f, 1.0f) * 255.0f + 0.5f)), 255);
}

// ---------------------------------------------------------------------------
// scene normals: 3x3x3 occupancy gradient of every leaf (normal.comp:73-95
// over the full cube), written into the leaf words' normal field.
// ---------------------------------------------------------------------------
// frontier entry: slot (28 bits) | x << 28 | y << 39 | z << 50 (11 bits each)
__device__ __forceinline__ unsigned long long pack_cell(uint32_t slot, uint32_t x, uint32_t y, uint32_t z) {
    return (unsigned long long)slot | ((unsigned long long)x << 28) | ((unsigned long long)y << 39) |
           ((unsigned long long)z << 50);
}

// Expands internal nodes of level k (cell size 2^(D-k)) into their internal
// children (level k+1).
__global__ void __launch_bounds__(256) k_expand(const uint32_t* __restrict__ nodes, uint64_t n_words, uint32_t D,
                                                uint32_t k, const unsigned long long* in, const uint32_t* in_cnt,
                                                unsigned long long* out, uint32_t* out_cnt, uint32_t cap) {
    const uint32_t n = min(*in_cnt, cap);
    const uint32_t half = (1u << D) >> (k + 1u);
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        unsigned long long e = 0;
        uint32_t word = 0;
        if (i < n) {
            e = in[i];
            word = fetch_node(nodes, n_words, uint32_t(e & 0xFFFFFFFull));
        }
        const uint32_t next = word >> 4;
        const uint32_t x = uint32_t((e >> 28) & 2047u), y = uint32_t((e >> 39) & 2047u), z = uint32_t((e >> 50) & 2047u);
        for (uint32_t c = 0; c < 8; c++) {
            bool app = false;
            if (i < n && (word & 1u)) app = (fetch_node(nodes, n_words, next + c) & 1u) != 0u;
            const uint32_t slot = warp_append(app, out_cnt);
            if (app && slot < cap)
                out[slot] = pack_cell(next + c, x + ((c & 4u) ? half : 0u), y + ((c & 2u) ? half : 0u),
                                      z + ((c & 1u) ? half : 0u));
        }
    }
}

__device__ __forceinline__ uint64_t occ_index(uint32_t x, uint32_t y, uint32_t z, uint32_t D) {
    return (((uint64_t(z) << D) + y) << D) + x;
}

// phase 0: set occupancy bits of all leaves below level D-1 nodes
// phase 1: compute and store the normal field of those leaves
__global__ void __launch_bounds__(256) k_leaf_pass(uint32_t* nodes, uint64_t n_words, uint32_t D,
                                                   const unsigned long long* in, const uint32_t* in_cnt,
                                                   uint32_t* occ, int phase, uint32_t cap) {
    const uint32_t n = min(*in_cnt, cap);
    const int L = int(1u << D);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const unsigned long long e = in[i];
        const uint32_t word = fetch_node(nodes, n_words, uint32_t(e & 0xFFFFFFFull));
        if (!(word & 1u)) continue;
        const uint32_t next = word >> 4;
        const uint32_t x0 = uint32_t((e >> 28) & 2047u), y0 = uint32_t((e >> 39) & 2047u),
                       z0 = uint32_t((e >> 50) & 2047u);
        for (uint32_t c = 0; c < 8; c++) {
            if (uint64_t(next) + c >= n_words) break;
            const uint32_t lw = nodes[next + c];
            if ((lw & 1u) || ((lw >> 1) & 0x7Fu) == 0u) continue;
            const uint32_t x = x0 + ((c >> 2) & 1u), y = y0 + ((c >> 1) & 1u), z = z0 + (c & 1u);
            if (phase == 0) {
                const uint64_t bi = occ_index(x, y, z, D);
                atomicOr(&occ[bi >> 5], 1u << (bi & 31u));
            } else {
                int ax = 0, ay = 0, az = 0;
                for (int dx = -1; dx <= 1; dx++)
                    for (int dy = -1; dy <= 1; dy++)
                        for (int dz = -1; dz <= 1; dz++) {
                            if (dx == 0 && dy == 0 && dz == 0) continue;
                            const int nx = int(x) + dx, ny = int(y) + dy, nz = int(z) + dz;
                            bool occd = false;
                            if (nx >= 0 && ny >= 0 && nz >= 0 && nx < L && ny < L && nz < L) {
                                const uint64_t bi = occ_index(uint32_t(nx), uint32_t(ny), uint32_t(nz), D);
                                occd = (occ[bi >> 5] >> (bi & 31u)) & 1u;
                            }
                            if (!occd) { ax += dx; ay += dy; az += dz; }
                        }
                nodes[next + c] = (lw & 0xFFu) | encode_normal_field(ax, ay, az);
            }
        }
    }
}

// The reference's own normal mode (normal.comp:55-95, computeRefinedNormal +
// packNormalAccum) for the leaves below each level-(D-1) node of `in`: the
// offsets d of the empty neighbours with 0 < |d|^2 <= R^2 around the voxel's
// even-aligned corner (the reference rebuilds the position from the
// GBuffer's half coordinates times two, normal.comp:147-152 — the corner of
// the level-(D-1) cell, shared by its 8 leaves), neighbours outside the
// volume counted as empty; normalize, or (0, 1, 0) when the sum vanishes; the
// 10-10-10 code is written at each leaf's slot of `codes`.  The sum is
// integer (exact), so its order does not matter.
__global__ void __launch_bounds__(256) k_ball_codes(const uint32_t* __restrict__ nodes, uint64_t n_words, uint32_t D,
                                                    const unsigned long long* in, const uint32_t* in_cnt,
                                                    const uint32_t* __restrict__ occ, int R, uint32_t* codes,
                                                    uint32_t cap) {
    const uint32_t n = min(*in_cnt, cap);
    const int L = int(1u << D);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const unsigned long long e = in[i];
        const uint32_t word = fetch_node(nodes, n_words, uint32_t(e & 0xFFFFFFFull));
        if (!(word & 1u)) continue;
        const uint32_t next = word >> 4;
        uint32_t leaves = 0;  // children that are leaves with a material
        for (uint32_t c = 0; c < 8u; c++) {
            if (uint64_t(next) + c >= n_words) break;
            const uint32_t lw = nodes[next + c];
            if (!(lw & 1u) && ((lw >> 1) & 0x7Fu) != 0u) leaves |= 1u << c;
        }
        if (!leaves) continue;
        const int x = int((e >> 28) & 2047u), y = int((e >> 39) & 2047u), z = int((e >> 50) & 2047u);
        int ax = 0, ay = 0, az = 0;
        for (int dx = -R; dx <= R; dx++)
            for (int dy = -R; dy <= R; dy++)
                for (int dz = -R; dz <= R; dz++) {
                    if ((dx | dy | dz) == 0 || dx * dx + dy * dy + dz * dz > R * R) continue;
                    const int nx = x + dx, ny = y + dy, nz = z + dz;
                    bool occd = false;
                    if (nx >= 0 && ny >= 0 && nz >= 0 && nx < L && ny < L && nz < L) {
                        const uint64_t bi = occ_index(uint32_t(nx), uint32_t(ny), uint32_t(nz), D);
                        occd = (__ldg(occ + (bi >> 5)) >> (bi & 31u)) & 1u;
                    }
                    if (!occd) { ax += dx; ay += dy; az += dz; }
                }
        const f3 acc = mk(float(ax), float(ay), float(az));
        const float len = sqrtf(dot(acc, acc));
        const f3 nv = len > 0.001f ? divs(acc, len) : mk(0.0f, 1.0f, 0.0f);
        const uint32_t code = (pack1022(nv.x) << 22) | (pack1022(nv.y) << 12) | (pack1022(nv.z) << 2);
        for (uint32_t c = 0; c < 8u; c++)
            if (leaves & (1u << c)) codes[next + c] = code;
    }
}

// UnpackNormal (internal.glsl:22-28) + normalize of every table code.
__global__ void __launch_bounds__(256) k_ball_table(const uint32_t* __restrict__ code, uint32_t n, float4* ntab) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t p = code[i];
        const f3 u = normalize(mk(float((p >> 22) & 0x3FFu) / 511.0f - 1.0f, float((p >> 12) & 0x3FFu) / 511.0f - 1.0f,
                                  float((p >> 2) & 0x3FFu) / 511.0f - 1.0f));
        ntab[i] = make_float4(u.x, u.y, u.z, 0.0f);
    }
}

// Each leaf's normal field := index + 1 of its code in the sorted table.
__global__ void __launch_bounds__(256) k_ball_apply(uint32_t* nodes, uint64_t n_words, const uint32_t* __restrict__ codes,
                                                    const uint32_t* __restrict__ table, uint32_t n) {
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n_words;
         i += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t code = codes[i];
        if (code == 0u) continue;
        uint32_t lo = 0, hi = n;  // first entry >= code
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (table[mid] < code) lo = mid + 1u; else hi = mid;
        }
        nodes[i] = (nodes[i] & 0xFFu) | ((lo + 1u) << 8);
    }
}

struct NonZero {
    __host__ __device__ bool operator()(uint32_t v) const { return v != 0u; }
};

// ---------------------------------------------------------------------------
// allocation-free leaf normal pass: its scratch lives in this fixed device
// array (the frontiers and the occupancy bitmask of a depth <= 7 scene),
// held by every GPU that loads the library until the process exits
// ---------------------------------------------------------------------------
constexpr uint32_t kNoAllocMaxDepth = 7;
constexpr uint64_t kNoAllocFrontier = 1ull << 18;  // 64^3: every size-2 cell of a depth-7 scene
constexpr uint64_t kNoAllocOccWords = (1ull << (3 * kNoAllocMaxDepth)) / 32;
constexpr size_t kNoAllocCounterBytes = 256;
constexpr size_t kNoAllocBytes = kNoAllocCounterBytes + 2 * kNoAllocFrontier * 8 + kNoAllocOccWords * 4;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// seeds the root frontier entry (slot 0, origin 0) and its count
__global__ void k_noalloc_seed(uint32_t* counters, unsigned long long* frontier) {
    if (threadIdx.x == 0) {
        counters[0] = 1u;
        frontier[0] = 0ull;
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static thread_local std::string g_err;
void set_last_error(const char* msg) { g_err = msg; }
static int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}
#define VE_CUDA(call)                                                                                   \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess)                                                                          \
            return fail(VE_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));               \
    } while (0)

struct SceneSlot {
    void* alloc = nullptr;   // node array allocation (nodes start 7 words in)
    uint32_t* nodes = nullptr;
    uint64_t n_words = 0;
    uint32_t depth = 0;
    CacheEntry* cache = nullptr;
    uint32_t* top = nullptr;  // top table of the DDA descent (see raycast.cuh)
    uint32_t top_level = 0;
    bool live = false;
    ve_nrc* nrc = nullptr;  // learned radiance cache attached to the scene
    float* rank = nullptr;  // scheduling state: {t_high, t_mid, histogram[256]}
    // emissive lights and ReSTIR reservoirs (allocated by the first emissive frame)
    ve::EmLight* em_list = nullptr;
    uint32_t* em_claim = nullptr;
    uint32_t* em_state = nullptr;
    ve::EmLight* em_stage = nullptr;
    ve::ResEntry* res = nullptr;
    uint32_t* lbuf = nullptr;  // dual-channel lBuffer (first VE_FRAME_LBUFFER frame)
    // normal mode: 0 = 3x3x3 occupancy gradient in the leaf words; R > 0 = the
    // reference's L2 ball of radius R, the leaf words indexing `ntab`
    uint32_t normal_radius = 0;
    float4* ntab = nullptr;
    uint32_t n_ntab = 0;
    // bounce-ray clip box (DevScene::clip_lo/hi), from the top table build;
    // unbounded when the scene has no top table
    float clip_lo[3] = {-1e30f, -1e30f, -1e30f}, clip_hi[3] = {1e30f, 1e30f, 1e30f};
};

template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t cap = 0;
    int ensure(size_t n) {
        if (n <= cap) return VE_OK;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        const size_t want = std::max<size_t>(n, 1);
        if (cudaMalloc(&p, want * sizeof(T)) != cudaSuccess)
            return fail(VE_ERR_NOMEM, "device allocation failed (" + std::to_string(want * sizeof(T)) + " bytes)");
        cap = want;
        return VE_OK;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
};

}  // namespace ve

// The buffers a plain frame's passes own, for the second of the two sets
// that pipelined frames (VE_CFG_PIPELINE) alternate between; the first set is
// the context's own members of the same names.
struct FrameSet {
    cudaStream_t stream = nullptr;
    ve::DevBuf<ve::DevView> d_views;
    ve::DevBuf<float4> p_ray_o, p_ray_d, p_tp, p_direct, p_indirect, p_pend;
    ve::DevBuf<uint4> p_hit, p_meta, gbuf;
    ve::DevBuf<uint32_t> live0, live1, counters;
    ve::DevBuf<uint2> rayq;
    ve::DevBuf<unsigned long long> stats;
    unsigned long long* h_stats = nullptr;  // pinned
};

struct ve_ctx {
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    ve_renderer_config cfg{};
    std::vector<ve::SceneSlot> scenes;
    ve::DevBuf<ve::DevScene> d_scenes;
    bool scenes_dirty = true;
    ve::DevBuf<ve::DevMaterial> d_mats;
    ve::DevBuf<ve::DevView> d_views;
    // pinned staging ring for the per-frame view table: a slot is rewritten
    // only after the copy that last read it has executed
    static constexpr int kStaging = 8;
    ve::DevView* h_views[kStaging] = {};
    size_t h_views_cap = 0;
    cudaEvent_t staging_ev[kStaging] = {};
    int staging_next = 0;
    ve::DevBuf<float4> p_ray_o, p_ray_d, p_tp, p_direct, p_indirect, p_pend;
    ve::DevBuf<uint4> p_hit, p_meta;
    ve::DevBuf<uint32_t> p_aux;  // training sample slot per path (learned-cache training frames)
    // importance-aware scheduling: primary hits, voxel claim table (key,
    // representative pixel, pixel count), per-pixel path counts and their
    // prefix sums, shade list, scan scratch
    ve::DevBuf<uint4> hitinfo;
    ve::DevBuf<uint32_t> claim, sched_n;
    ve::DevBuf<uint2> shade_list;
    ve::DevBuf<uint8_t> scan_tmp;
    ve::DevBuf<uint32_t> live0, live1;
    ve::DevBuf<uint2> rayq;
    ve::DevBuf<uint32_t> counters;
    ve::DevBuf<unsigned long long> stats;
    ve::DevBuf<unsigned long long> totals;
    unsigned long long* h_stats = nullptr;  // pinned
    // host-side running totals (ve_get_total_stats)
    uint64_t tot_frames = 0, tot_h2d = 0, tot_d2h = 0;
    uint32_t tot_launches = 0, tot_trace_launches = 0;
    float tot_ms[6] = {0, 0, 0, 0, 0, 0};
    float tot_ms_learned = 0;
    uint64_t last_h2d = 0, last_d2h = 0;
    ve::DevBuf<uint4> gbuf;
    ve::DevBuf<uint32_t> out_vid, out_node;
    ve::DevBuf<float> out_rgb, out_mapped, path_rgb;
    ve::DevBuf<uchar4> out_m8;
    // VE_FRAME_ASYNC_OUTPUTS: a second set of device images (frames alternate
    // between the sets), the stream their host copies run on, and events
    // that order a set's next resolve after its last copy
    ve::DevBuf<uint32_t> out_vid2, out_node2;
    ve::DevBuf<float> out_rgb2, out_mapped2;
    ve::DevBuf<uchar4> out_m82;
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t frame_done = nullptr, copy_done[2] = {};
    int out_parity = 0;
    // VE_CFG_PIPELINE: the second frame set and the order between the sets.
    // A pipelined frame's primary and first trace pass touch only its own
    // set, so they run while the other set's frame finishes; its cache work
    // (decay, deposits, AvgPass) waits for that frame's (set_cache_done).
    FrameSet alt;
    int pipe_next = 0;           // set of the next pipelined frame
    int last_set = 0;            // set that rendered the last frame (its stats)
    bool alt_busy = false;       // work of the second set may be in flight
    bool ops_pending = false;    // main-stream work enqueued since the last second-set frame
    cudaEvent_t set_cache_done[2] = {};  // end of each set's last frame's cache work
    cudaEvent_t alt_done = nullptr;      // end of the last second-set frame
    cudaEvent_t ops_ev = nullptr;        // main-stream point a second-set frame waits for
    ve::DevBuf<float4> p_sdir;          // emissive batches: NEE shadow directions + light vid
    ve::DevBuf<ve::PathRes> p_res;      // emissive batches: bounce-0 reservoirs until the commit
    ve::DevBuf<uint32_t> res_list;      // ... and the paths that hold one
    ve::DevBuf<uint32_t> em_sort;       // registry commit: vid keys / staging indices, 2 x 2 x 2^17
    ve::DevBuf<uint8_t> em_sort_tmp;    // ... CUB radix-sort scratch
    ve::DevBuf<ve::LbRec> lb_rec;        // lBuffer frames: deposits at their path slots
    ve::DevBuf<uint32_t> lb_keys;        // ... their rows (0: none), 2 x paths (sort in, out)
    ve::DevBuf<uint32_t> lb_idx;         // ... path slots 0..n-1 (sort values in), order (out), row bounds
    ve::DevBuf<uint8_t> lb_tmp;          // ... CUB radix-sort scratch
    uint64_t lb_iota = 0;                // lb_idx holds 0..lb_iota-1
    // split frames: the per-frame deposit table, the scene table whose
    // cache points at it, export / merge counters, the scene of the last
    // split frame
    ve::DevBuf<ve::CacheEntry> split_delta;
    ve::DevBuf<ve::DevScene> d_scenes_split;
    ve::DevBuf<uint32_t> split_cnt;
    int split_scene = -1;
    bool split_delta_clean = false;  // the per-frame table is all zeros (cleared by the last export)
    ve_frame_config split_frame{};  // the last split frame's config
    ve::DevBuf<float> ray_in;      // ve_raycast_batch: origins and directions
    ve::DevBuf<uint32_t> ray_out;  // ve_raycast_batch: 8 words per ray
    int grid_trace = 0, grid_trace_count = 0, grid_shade = 0;
    int occ_trace = 1, occ_trace_count = 1, occ_shade = 1;  // occupancy maxima (blocks/SM)
    int occ_shade_mode[8] = {1, 1, 1, 1, 1, 1, 1, 1};       // ... per shading instance (kModeEm | kModeLb | kModeNrc)
    int occ_emit_mode[4] = {1, 1, 1, 1};                    // ... per scheduled-emit instance
    ve_launch_config launch{0, 0, ve::kDefaultRefill, 0};
    // per-frame CUDA-event sets in a ring: elapsed times are read when the
    // slot is reused or the stats are queried, so timed frames never wait
    static constexpr int kTimingSlots = 16, kEvents = 48;
    struct TimingSlot {
        cudaEvent_t ev[kEvents] = {};
        int n = 0;            // events recorded
        uint32_t passes = 0;  // shade passes
        bool learned = false; // a learned-cache segment precedes resolve
        bool pending = false;
    } timing[kTimingSlots];
    int timing_next = 0;
    ve_frame_stats last{};
    bool last_timing = false;
    int last_timing_slot = -1;
    // CUDA graphs of the per-frame kernel sequence, keyed by what shapes it;
    // `gen` changes whenever a buffer or scene the kernels point at moves
    uint64_t gen = 1;
    struct GraphEntry {
        std::vector<uint64_t> key;
        cudaGraphExec_t exec = nullptr;
        uint32_t launches = 0, trace_launches = 0;
        uint64_t last_use = 0;
    };
    std::vector<GraphEntry> graphs;
    uint64_t graph_clock = 0;
    uint64_t graph_captures = 0, graph_replays = 0;
    std::vector<ve_nrc*> nrcs;  // learned caches created on this context
    uint32_t last_launches = 0, last_trace_launches = 0;
};

namespace ve {
namespace nrc {
static int set_frame_infer_attributes() {
    if (cudaFuncSetAttribute(k_nrc_infer<ApplyDeposit>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(kSmemInfer)) != cudaSuccess)
        return VE_ERR_CUDA;
    cudaFuncSetAttribute(k_nrc_infer<ApplyDeposit>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    return VE_OK;
}
}  // namespace nrc
static void join_alt(ve_ctx* c);
}  // namespace ve

#include "nrc_host.cuh"

namespace ve {

static int sync_scenes(ve_ctx* c) {
    if (!c->scenes_dirty) return VE_OK;
    std::vector<DevScene> h(std::max<size_t>(c->scenes.size(), 1));
    for (size_t i = 0; i < c->scenes.size(); i++) {
        const SceneSlot& s = c->scenes[i];
        h[i] = DevScene{s.nodes,     s.n_words,   s.cache,    s.depth,    c->cfg.hash_log2, c->cfg.hash_probes,
                        s.top_level, s.top,       s.em_list, s.em_claim, s.em_state,       s.em_stage,
                        s.res,       s.lbuf,      s.ntab,    s.n_ntab,
                        {s.clip_lo[0], s.clip_lo[1], s.clip_lo[2]},
                        {s.clip_hi[0], s.clip_hi[1], s.clip_hi[2]}};
    }
    const void* old = c->d_scenes.p;
    int rc = c->d_scenes.ensure(h.size());
    if (rc) return rc;
    if (old != c->d_scenes.p) c->gen++;
    VE_CUDA(cudaMemcpyAsync(c->d_scenes.p, h.data(), h.size() * sizeof(DevScene), cudaMemcpyHostToDevice, c->stream));
    VE_CUDA(cudaStreamSynchronize(c->stream));
    c->scenes_dirty = false;
    return VE_OK;
}

// Top table of the DDA descent: one word per cell of the level-(T0-1) grid,
// found by walking levels 0..T0-1 of the node words exactly as the descent
// does (out-of-range words read as zero).
//
// Also the box of the cells that can hold a voxel: a descent that ends above
// level D steps over an empty cell (only level-D words are tested for a
// material), so only cells internal down to level T0 can be hit.  box[0..2]
// = smallest, box[3..5] = largest such cell coordinate (box[0] > box[3]: no
// such cell).  Positions with a coordinate equal to 2^D lie outside the
// table; k_face_hits covers them.
__global__ void k_build_top(const uint32_t* __restrict__ nodes, uint64_t n_words, uint32_t D, uint32_t T0,
                            uint32_t* __restrict__ top, uint32_t* __restrict__ box) {
    __shared__ uint32_t sb[6];
    if (threadIdx.x < 6) sb[threadIdx.x] = threadIdx.x < 3 ? 0xFFFFFFFFu : 0u;
    const uint32_t b = T0 - 1u, n = 1u << (3u * b);
    const uint32_t sh = D - T0 + 1u, L = 1u << D;
    uint32_t lo[3] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu}, hi[3] = {0u, 0u, 0u};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t cx = i >> (2u * b), cy = (i >> b) & ((1u << b) - 1u), cz = i & ((1u << b) - 1u);
        const uint32_t x = cx << sh, y = cy << sh, z = cz << sh;
        uint32_t base = 0, ent = 0;
        bool terminal = false;
        for (uint32_t k = 0; k < T0; k++) {
            const uint32_t raw = dev::fetch_node(nodes, n_words, base + locate(x, y, z, L >> k));
            if (!(raw & 1u)) {
                ent = k << 1;
                terminal = true;
                break;
            }
            base = raw >> 4;
        }
        top[i] = terminal ? ent : ((base << 1) | 1u);
        if (!terminal) {
            lo[0] = min(lo[0], cx); lo[1] = min(lo[1], cy); lo[2] = min(lo[2], cz);
            hi[0] = max(hi[0], cx); hi[1] = max(hi[1], cy); hi[2] = max(hi[2], cz);
        }
    }
    __syncthreads();
    for (int a = 0; a < 3; a++) {
        const uint32_t wl = __reduce_min_sync(0xFFFFFFFFu, lo[a]), wh = __reduce_max_sync(0xFFFFFFFFu, hi[a]);
        if ((threadIdx.x & 31u) == 0u) {
            atomicMin(&sb[a], wl);
            atomicMax(&sb[3 + a], wh);
        }
    }
    __syncthreads();
    if (threadIdx.x < 3) atomicMin(&box[threadIdx.x], sb[threadIdx.x]);
    else if (threadIdx.x < 6) atomicMax(&box[threadIdx.x], sb[threadIdx.x]);
}

// The DDA's bounds test admits a coordinate equal to 2^D, whose bit D sends
// the level-0 read to root words 1..7 instead of word 0 (internal.glsl's
// locate at octreeLength).  Sets *hit when any integer position on the three
// faces {x, y or z = 2^D} ends its descent on a material voxel — the only
// positions outside the top table's cells that can be hit.
__global__ void __launch_bounds__(256) k_face_hits(const uint32_t* __restrict__ nodes, uint64_t n_words, uint32_t D,
                                                   uint32_t* hit) {
    const uint32_t L = 1u << D, side = L + 1u;
    const uint64_t per_face = uint64_t(side) * side;
    bool any = false;
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < 3u * per_face;
         i += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t f = uint32_t(i / per_face);
        const uint64_t j = i % per_face;
        const uint32_t u = uint32_t(j / side), v = uint32_t(j % side);
        const uint32_t x = f == 0 ? L : u, y = f == 1 ? L : (f == 0 ? u : v), z = f == 2 ? L : v;
        // the descent of dda_step without the top table
        uint32_t base = 0;
        bool internal = true;
        for (uint32_t k = 0; k < D && internal; k++) {
            const uint32_t b = D - k;
            const uint32_t raw = dev::fetch_node(nodes, n_words,
                                                 base + ((((x >> b) & 1u) << 2) | (((y >> b) & 1u) << 1) | ((z >> b) & 1u)));
            internal = (raw & 1u) != 0u;
            base = raw >> 4;
        }
        if (internal) {
            const uint32_t raw = dev::fetch_node(nodes, n_words, base + (((x & 1u) << 2) | ((y & 1u) << 1) | (z & 1u)));
            any |= ((raw & 254u) >> 1) != 0u;
        }
    }
    if (__any_sync(0xFFFFFFFFu, any) && (threadIdx.x & 31u) == 0u) atomicOr(hit, 1u);
}

// Octree::applyEdits upload (octree.cpp:228-314): words[i] -> nodes[slots[i]].
__global__ void k_scatter_words(uint32_t* __restrict__ nodes, const uint32_t* __restrict__ slots,
                                const uint32_t* __restrict__ words, uint64_t n) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
        nodes[slots[i]] = words[i];
}

// Slot of the voxel leaf at (x, y, z) when it holds a material, else ~0u:
// the descent of the DDA (internal words down to level D, leaf word there).
__device__ __forceinline__ uint32_t leaf_slot(const uint32_t* __restrict__ nodes, uint64_t n_words, uint32_t D,
                                              uint32_t x, uint32_t y, uint32_t z) {
    const uint32_t L = 1u << D;
    uint32_t base = 0;
    for (uint32_t k = 0; k < D; k++) {
        const uint32_t raw = dev::fetch_node(nodes, n_words, base + locate(x, y, z, L >> k));
        if (!(raw & 1u)) return ~0u;
        base = raw >> 4;
    }
    const uint32_t slot = base + locate(x, y, z, 1u);
    const uint32_t raw = dev::fetch_node(nodes, n_words, slot);
    return (!(raw & 1u) && ((raw >> 1) & 0x7Fu) != 0u) ? slot : ~0u;
}

// Targeted refresh after an edit: for every voxel of the 3x3x3 neighbourhood
// of each edited position, the leaf normal field (the full pass's 26-
// neighbour gradient of the occupancy, k_leaf_pass) and, when `cache` is
// given, the radiance-cache entry (sums, weight and count cleared, key kept
// so probe chains stay intact).  Normal writes keep bits 0-7, the only bits
// the concurrent occupancy lookups read.
__global__ void k_refresh(uint32_t* __restrict__ nodes, uint64_t n_words, uint32_t D, const uint32_t* __restrict__ xyz,
                          uint64_t n, CacheEntry* cache, uint32_t cache_log2, uint32_t probes) {
    const int L = int(1u << D);
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n * 27u;
         i += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t e = i / 27u;
        const int o = int(i % 27u);
        const int x = int(xyz[3 * e]) + o / 9 - 1, y = int(xyz[3 * e + 1]) + (o / 3) % 3 - 1, z = int(xyz[3 * e + 2]) + o % 3 - 1;
        if (x < 0 || y < 0 || z < 0 || x >= L || y >= L || z >= L) continue;
        if (cache) {
            const int c = cache_find(cache, cache_log2, probes, voxel_key(uint32_t(x), uint32_t(y), uint32_t(z)) + 1u);
            if (c >= 0) {
                cache[c].count = 0u;
                cache[c].l2 = 0.0f;
                cache[c].rgbw = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            }
        }
        const uint32_t slot = leaf_slot(nodes, n_words, D, uint32_t(x), uint32_t(y), uint32_t(z));
        if (slot == ~0u) continue;
        int ax = 0, ay = 0, az = 0;
        for (int dx = -1; dx <= 1; dx++)
            for (int dy = -1; dy <= 1; dy++)
                for (int dz = -1; dz <= 1; dz++) {
                    if (dx == 0 && dy == 0 && dz == 0) continue;
                    const int nx = x + dx, ny = y + dy, nz = z + dz;
                    bool occd = false;
                    if (nx >= 0 && ny >= 0 && nz >= 0 && nx < L && ny < L && nz < L)
                        occd = leaf_slot(nodes, n_words, D, uint32_t(nx), uint32_t(ny), uint32_t(nz)) != ~0u;
                    if (!occd) {
                        ax += dx;
                        ay += dy;
                        az += dz;
                    }
                }
        const uint32_t lw = nodes[slot];
        nodes[slot] = (lw & 0xFFu) | encode_normal_field(ax, ay, az);
    }
}

// Levels resolved by the top table: every level above the leaves up to
// depth 10 (levels 0..D-1: a descent is one table word, then the leaf word),
// levels 0..9 deeper down, none under depth 3.  At depth 10 the table is
// 512^3 words (512 MiB): trace 1.084 -> 1.017 ms per 1080p frame against
// levels 0..8 (256^3 words), which in turn beat levels 0..7 (1.54 -> 1.43).
static uint32_t top_levels(uint32_t D) { return D < 3u ? 0u : std::min(10u, D); }

static int build_top(ve_ctx* c, SceneSlot& s) {
    const uint32_t T0 = top_levels(s.depth);
    c->scenes_dirty = true;
    for (int a = 0; a < 3; a++) {  // unbounded until the table says otherwise
        s.clip_lo[a] = -1e30f;
        s.clip_hi[a] = 1e30f;
    }
    if (T0 == 0) return VE_OK;
    const size_t n = size_t(1) << (3u * (T0 - 1u));
    if (!s.top) {
        if (cudaMalloc(&s.top, n * 4) != cudaSuccess) return fail(VE_ERR_NOMEM, "scene: top table allocation failed");
    }
    s.top_level = T0;
    uint32_t* d_box = nullptr;
    if (cudaMalloc(&d_box, 7 * 4) != cudaSuccess) return fail(VE_ERR_NOMEM, "scene: allocation failed");
    const uint32_t init[7] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0u, 0u, 0u, 0u};
    uint32_t box[7];
    cudaMemcpyAsync(d_box, init, sizeof(init), cudaMemcpyHostToDevice, c->stream);
    k_build_top<<<c->num_sms * 8, 256, 0, c->stream>>>(s.nodes, s.n_words, s.depth, T0, s.top, d_box);
    // faces of more than 3 * 4097^2 positions are not searched: no box then
    if (s.depth <= 12) k_face_hits<<<c->num_sms * 8, 256, 0, c->stream>>>(s.nodes, s.n_words, s.depth, d_box + 6);
    cudaMemcpyAsync(box, d_box, sizeof(box), cudaMemcpyDeviceToHost, c->stream);
    const cudaError_t e = cudaStreamSynchronize(c->stream);
    cudaFree(d_box);
    if (e != cudaSuccess) return fail(VE_ERR_CUDA, std::string("scene: top table build: ") + cudaGetErrorString(e));
    if (s.depth > 12) box[6] = 1u;
    if (!box[6]) {
        // cells are 2^(D-T0+1) voxels wide; one voxel of margin on each side
        // keeps the box conservative against rounding of the ray positions
        const uint32_t sh = s.depth - T0 + 1u;
        for (int a = 0; a < 3; a++) {
            if (box[0] > box[3]) {  // no cell can be hit: any box is exact
                s.clip_lo[a] = -1.0f;
                s.clip_hi[a] = 1.0f;
            } else {
                s.clip_lo[a] = float(box[a] << sh) - 1.0f;
                s.clip_hi[a] = float((box[3 + a] + 1u) << sh) + 1.0f;
            }
        }
    }
    return VE_OK;
}

static int compute_normals(ve_ctx* c, SceneSlot& s) {
    const uint32_t D = s.depth;
    if (D < 1 || D > 11) return VE_OK;
    const uint64_t cap = std::max<uint64_t>(s.n_words, 16);
    unsigned long long *fa = nullptr, *fb = nullptr;
    uint32_t* cnt = nullptr;
    uint32_t* occ = nullptr;
    const uint64_t occ_words = ((1ull << (3 * D)) + 31) / 32;
    auto cleanup = [&]() {
        if (fa) cudaFree(fa);
        if (fb) cudaFree(fb);
        if (cnt) cudaFree(cnt);
        if (occ) cudaFree(occ);
    };
    if (cudaMalloc(&fa, cap * 8) != cudaSuccess || cudaMalloc(&fb, cap * 8) != cudaSuccess ||
        cudaMalloc(&cnt, 64 * 4) != cudaSuccess || cudaMalloc(&occ, occ_words * 4) != cudaSuccess) {
        cleanup();
        return fail(VE_ERR_NOMEM, "normal pass: device allocation failed");
    }
    cudaMemsetAsync(cnt, 0, 64 * 4, c->stream);
    cudaMemsetAsync(occ, 0, occ_words * 4, c->stream);
    const unsigned long long root = 0ull;  // slot 0, origin (0,0,0), level 0
    cudaMemcpyAsync(fa, &root, 8, cudaMemcpyHostToDevice, c->stream);
    const uint32_t one = 1;
    cudaMemcpyAsync(cnt, &one, 4, cudaMemcpyHostToDevice, c->stream);
    const int grid = c->num_sms * 8;
    unsigned long long* in = fa;
    unsigned long long* out = fb;
    for (uint32_t k = 0; k + 1 < D; k++) {
        k_expand<<<grid, 256, 0, c->stream>>>(s.nodes, s.n_words, D, k, in, cnt + k, out, cnt + k + 1,
                                              uint32_t(cap));
        std::swap(in, out);
    }
    const uint32_t* lc = cnt + (D - 1);
    k_leaf_pass<<<grid, 256, 0, c->stream>>>(s.nodes, s.n_words, D, in, lc, occ, 0, uint32_t(cap));
    if (s.normal_radius == 0u) {
        k_leaf_pass<<<grid, 256, 0, c->stream>>>(s.nodes, s.n_words, D, in, lc, occ, 1, uint32_t(cap));
        cudaError_t e = cudaStreamSynchronize(c->stream);
        cleanup();
        if (e != cudaSuccess) return fail(VE_ERR_CUDA, std::string("normal pass: ") + cudaGetErrorString(e));
        if (s.ntab) {  // back from the ball mode
            cudaFree(s.ntab);
            s.ntab = nullptr;
            s.n_ntab = 0;
            c->scenes_dirty = true;
        }
        return VE_OK;
    }
    // the reference's ball mode: a code per leaf, then the sorted table of
    // distinct codes, and every leaf's index into it
    if (s.n_words > uint64_t(INT32_MAX)) {
        cleanup();
        return fail(VE_ERR_CAPACITY, "normal pass (ball): more than 2^31 words");
    }
    const int nw = int(s.n_words);
    uint32_t *codes = nullptr, *sel = nullptr, *table = nullptr, *nsel = nullptr;
    void* tmp = nullptr;
    auto cleanup2 = [&]() {
        cleanup();
        for (void* p : {(void*)codes, (void*)sel, (void*)table, (void*)nsel, tmp})
            if (p) cudaFree(p);
    };
    size_t b_sel = 0, b_sort = 0, b_uniq = 0;
    cub::DeviceSelect::If(nullptr, b_sel, codes, sel, nsel, nw, NonZero(), c->stream);
    cub::DeviceRadixSort::SortKeys(nullptr, b_sort, sel, table, nw, 2, 32, c->stream);
    cub::DeviceSelect::Unique(nullptr, b_uniq, table, sel, nsel + 1, nw, c->stream);
    const size_t b_tmp = std::max(b_sel, std::max(b_sort, b_uniq));
    if (cudaMalloc(&codes, size_t(nw) * 4) != cudaSuccess || cudaMalloc(&sel, size_t(nw) * 4) != cudaSuccess ||
        cudaMalloc(&table, size_t(nw) * 4) != cudaSuccess || cudaMalloc(&nsel, 2 * 4) != cudaSuccess ||
        cudaMalloc(&tmp, std::max<size_t>(b_tmp, 16)) != cudaSuccess) {
        cleanup2();
        return fail(VE_ERR_NOMEM, "normal pass (ball): device allocation failed");
    }
    cudaMemsetAsync(codes, 0, size_t(nw) * 4, c->stream);
    k_ball_codes<<<grid, 256, 0, c->stream>>>(s.nodes, s.n_words, D, in, lc, occ, int(s.normal_radius), codes,
                                              uint32_t(cap));
    uint32_t h_n[2] = {0, 0};
    size_t bt = b_tmp;
    cub::DeviceSelect::If(tmp, bt, codes, sel, nsel, nw, NonZero(), c->stream);
    cudaMemcpyAsync(&h_n[0], nsel, 4, cudaMemcpyDeviceToHost, c->stream);
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e == cudaSuccess && h_n[0] > 0u) {
        bt = b_tmp;
        cub::DeviceRadixSort::SortKeys(tmp, bt, sel, table, int(h_n[0]), 2, 32, c->stream);
        bt = b_tmp;
        cub::DeviceSelect::Unique(tmp, bt, table, sel, nsel + 1, int(h_n[0]), c->stream);
        cudaMemcpyAsync(&h_n[1], nsel + 1, 4, cudaMemcpyDeviceToHost, c->stream);
        e = cudaStreamSynchronize(c->stream);
    }
    if (e != cudaSuccess) {
        cleanup2();
        return fail(VE_ERR_CUDA, std::string("normal pass (ball): ") + cudaGetErrorString(e));
    }
    if (s.ntab) cudaFree(s.ntab);
    s.ntab = nullptr;
    s.n_ntab = 0;
    if (h_n[1] > 0u) {
        if (cudaMalloc(&s.ntab, size_t(h_n[1]) * sizeof(float4)) != cudaSuccess) {
            s.ntab = nullptr;
            cleanup2();
            return fail(VE_ERR_NOMEM, "normal pass (ball): table allocation failed");
        }
        s.n_ntab = h_n[1];
        k_ball_table<<<grid, 256, 0, c->stream>>>(sel, h_n[1], s.ntab);
        k_ball_apply<<<grid, 256, 0, c->stream>>>(s.nodes, s.n_words, codes, sel, h_n[1]);
    }
    e = cudaStreamSynchronize(c->stream);
    cleanup2();
    c->scenes_dirty = true;
    if (e != cudaSuccess) return fail(VE_ERR_CUDA, std::string("normal pass (ball): ") + cudaGetErrorString(e));
    return VE_OK;
}

// Scheduling thresholds {t_high = +inf, t_mid = -inf} and an empty histogram:
// every voxel of the next scheduled frame falls in the middle tier.
constexpr size_t kLbBytes = size_t(kLbWidth) * kLbRowWords * sizeof(uint32_t);

static int ensure_lbuffer(ve_ctx* c, SceneSlot& s) {
    if (s.lbuf) return VE_OK;
    if (cudaMalloc(&s.lbuf, kLbBytes) != cudaSuccess) {
        s.lbuf = nullptr;
        return fail(VE_ERR_NOMEM, "render: lBuffer allocation failed");
    }
    VE_CUDA(cudaMemsetAsync(s.lbuf, 0, kLbBytes, c->stream));
    VE_CUDA(cudaStreamSynchronize(c->stream));
    c->scenes_dirty = true;
    return VE_OK;
}

static void free_emissive(SceneSlot& s) {
    if (s.em_list) cudaFree(s.em_list);
    if (s.em_claim) cudaFree(s.em_claim);
    if (s.em_state) cudaFree(s.em_state);
    if (s.em_stage) cudaFree(s.em_stage);
    if (s.res) cudaFree(s.res);
    s.em_list = nullptr;
    s.em_claim = nullptr;
    s.em_state = nullptr;
    s.em_stage = nullptr;
    s.res = nullptr;
}

// No lights registered or staged, no reservoirs.
static int reset_emissive(ve_ctx* c, SceneSlot& s) {
    if (!s.em_claim) return VE_OK;
    VE_CUDA(cudaMemsetAsync(s.em_claim, 0, sizeof(uint32_t) << kEmClaimLog2, c->stream));
    VE_CUDA(cudaMemsetAsync(s.em_state, 0, 2 * sizeof(uint32_t), c->stream));
    VE_CUDA(cudaMemsetAsync(s.res, 0, sizeof(ResEntry) << kResLog2, c->stream));
    VE_CUDA(cudaStreamSynchronize(c->stream));
    return VE_OK;
}

// The scene's light registry and reservoir table (first emissive frame).
static int ensure_emissive(ve_ctx* c, SceneSlot& s) {
    if (s.em_claim) return VE_OK;
    if (cudaMalloc(&s.em_list, sizeof(EmLight) * kEmCapacity) != cudaSuccess ||
        cudaMalloc(&s.em_claim, sizeof(uint32_t) << kEmClaimLog2) != cudaSuccess ||
        cudaMalloc(&s.em_state, 2 * sizeof(uint32_t)) != cudaSuccess ||
        cudaMalloc(&s.em_stage, sizeof(EmLight) << kEmClaimLog2) != cudaSuccess ||
        cudaMalloc(&s.res, sizeof(ResEntry) << kResLog2) != cudaSuccess) {
        free_emissive(s);
        return fail(VE_ERR_NOMEM, "render: emissive-light state allocation failed");
    }
    c->scenes_dirty = true;
    return reset_emissive(c, s);
}

static int reset_rank(ve_ctx* c, float* rank) {
    std::vector<uint32_t> init(2 + kRankBins, 0u);
    init[0] = 0x7f800000u;
    init[1] = 0xff800000u;
    VE_CUDA(cudaMemcpyAsync(rank, init.data(), init.size() * 4, cudaMemcpyHostToDevice, c->stream));
    VE_CUDA(cudaStreamSynchronize(c->stream));
    return VE_OK;
}

// Exchanges the context's first-set frame buffers (and stream) with the
// second set's: while swapped, the frame code's c->... members are set 1.
static void swap_set(ve_ctx* c) {
    FrameSet& a = c->alt;
    std::swap(c->stream, a.stream);
    std::swap(c->d_views, a.d_views);
    std::swap(c->p_ray_o, a.p_ray_o); std::swap(c->p_ray_d, a.p_ray_d); std::swap(c->p_tp, a.p_tp);
    std::swap(c->p_direct, a.p_direct); std::swap(c->p_indirect, a.p_indirect); std::swap(c->p_pend, a.p_pend);
    std::swap(c->p_hit, a.p_hit); std::swap(c->p_meta, a.p_meta); std::swap(c->gbuf, a.gbuf);
    std::swap(c->live0, a.live0); std::swap(c->live1, a.live1); std::swap(c->rayq, a.rayq);
    std::swap(c->counters, a.counters);
    std::swap(c->stats, a.stats);
    std::swap(c->h_stats, a.h_stats);
}

// Set 1 swapped in for the scope (a frame of the second set).
struct SetScope {
    ve_ctx* c;
    bool on;
    SetScope(ve_ctx* cc, bool use) : c(cc), on(use) {
        if (on) swap_set(c);
    }
    ~SetScope() {
        if (on) swap_set(c);
    }
};

// Orders work enqueued next on the main stream after every second-set frame
// in flight, and the next second-set frame after that work.  Every entry
// point that enqueues on the context's stream, other than a pipelined frame,
// calls it first.
static void join_alt(ve_ctx* c) {
    if (c->alt_busy) {
        cudaStreamWaitEvent(c->stream, c->alt_done, 0);
        c->alt_busy = false;
    }
    c->ops_pending = true;
}

static int ensure_frame(ve_ctx* c, uint64_t pixels, uint64_t paths, uint32_t n_views) {
    int rc = 0;
    const void* before[] = {c->gbuf.p, c->out_vid.p, c->out_node.p, c->out_rgb.p, c->out_mapped.p, c->out_m8.p,
                            c->p_ray_o.p, c->p_ray_d.p, c->p_tp.p, c->p_direct.p, c->p_indirect.p, c->p_pend.p,
                            c->p_hit.p, c->p_meta.p, c->live0.p, c->live1.p, c->rayq.p, c->d_views.p};
    struct GenBump {
        ve_ctx* c;
        const void* const* before;
        ~GenBump() {
            const void* after[] = {c->gbuf.p, c->out_vid.p, c->out_node.p, c->out_rgb.p, c->out_mapped.p,
                                   c->out_m8.p, c->p_ray_o.p, c->p_ray_d.p, c->p_tp.p, c->p_direct.p, c->p_indirect.p,
                                   c->p_pend.p, c->p_hit.p, c->p_meta.p, c->live0.p, c->live1.p,
                                   c->rayq.p, c->d_views.p};
            for (size_t i = 0; i < sizeof(after) / sizeof(after[0]); i++)
                if (after[i] != before[i]) { c->gen++; break; }
        }
    } bump{c, before};
    // a copy of an earlier frame's images may still read the buffers
    if (c->copy_stream && (pixels > c->out_vid.cap || 3 * pixels > c->out_rgb.cap))
        cudaStreamSynchronize(c->copy_stream);
    if ((rc = c->gbuf.ensure(pixels)) || (rc = c->out_vid.ensure(pixels)) || (rc = c->out_node.ensure(pixels)) ||
        (rc = c->out_rgb.ensure(pixels * 3)) || (rc = c->out_mapped.ensure(pixels * 3)) ||
        (rc = c->out_m8.ensure(pixels)))
        return rc;
    if ((rc = c->p_ray_o.ensure(paths)) || (rc = c->p_ray_d.ensure(paths)) || (rc = c->p_tp.ensure(paths)) ||
        (rc = c->p_direct.ensure(paths)) || (rc = c->p_indirect.ensure(paths)) || (rc = c->p_pend.ensure(paths)) ||
        (rc = c->p_hit.ensure(paths)) || (rc = c->p_meta.ensure(paths)) ||
        (rc = c->live0.ensure(paths)) || (rc = c->live1.ensure(paths)) || (rc = c->rayq.ensure(paths * 2)))
        return rc;
    if ((rc = c->d_views.ensure(n_views))) return rc;
    if (c->h_views_cap < n_views) {
        cudaStreamSynchronize(c->stream);
        for (int k = 0; k < ve_ctx::kStaging; k++) {
            if (c->h_views[k]) cudaFreeHost(c->h_views[k]);
            c->h_views[k] = nullptr;
            if (cudaMallocHost(&c->h_views[k], sizeof(DevView) * n_views) != cudaSuccess)
                return fail(VE_ERR_NOMEM, "pinned view table allocation failed");
        }
        c->h_views_cap = n_views;
    }
    return VE_OK;
}

// Reads one frame's event set (waits for its last event) and adds it to the
// running totals; `out` receives the frame's own stage times when non-null.
static void collect_timing(ve_ctx* c, ve_ctx::TimingSlot& ts, ve_frame_stats* out) {
    if (!ts.pending) return;
    cudaEventSynchronize(ts.ev[ts.n - 1]);
    ve_frame_stats f{};
    float t = 0;
    cudaEventElapsedTime(&t, ts.ev[0], ts.ev[1]); f.ms_decay = t;
    cudaEventElapsedTime(&t, ts.ev[1], ts.ev[2]); f.ms_primary = t;
    for (uint32_t pass = 0; pass < ts.passes; pass++) {
        const int e0 = 2 + 2 * int(pass);
        cudaEventElapsedTime(&t, ts.ev[e0], ts.ev[e0 + 1]); f.ms_shade += t;
        cudaEventElapsedTime(&t, ts.ev[e0 + 1], ts.ev[e0 + 2]); f.ms_trace += t;
    }
    cudaEventElapsedTime(&t, ts.ev[ts.n - 2], ts.ev[ts.n - 1]); f.ms_resolve = t;
    if (ts.learned) {
        cudaEventElapsedTime(&t, ts.ev[ts.n - 3], ts.ev[ts.n - 2]);
        f.ms_learned = t;
    }
    cudaEventElapsedTime(&t, ts.ev[0], ts.ev[ts.n - 1]); f.ms_total = t;
    c->tot_ms[0] += f.ms_total; c->tot_ms[1] += f.ms_primary; c->tot_ms[2] += f.ms_trace;
    c->tot_ms[3] += f.ms_shade; c->tot_ms[4] += f.ms_resolve; c->tot_ms[5] += f.ms_decay;
    ts.pending = false;
    c->tot_ms_learned += f.ms_learned;
    if (out) {
        out->ms_total = f.ms_total; out->ms_primary = f.ms_primary; out->ms_trace = f.ms_trace;
        out->ms_shade = f.ms_shade; out->ms_resolve = f.ms_resolve; out->ms_decay = f.ms_decay;
        out->ms_learned = f.ms_learned;
    }
}

static void collect_all_timing(ve_ctx* c) {
    for (int i = 0; i < ve_ctx::kTimingSlots; i++) {
        const int k = (c->timing_next + i) % ve_ctx::kTimingSlots;
        if (c->timing[k].pending) {
            ve_frame_stats f{};
            collect_timing(c, c->timing[k], &f);
            if (k == c->last_timing_slot) {
                c->last.ms_total = f.ms_total; c->last.ms_primary = f.ms_primary; c->last.ms_trace = f.ms_trace;
                c->last.ms_shade = f.ms_shade; c->last.ms_resolve = f.ms_resolve; c->last.ms_decay = f.ms_decay;
                c->last.ms_learned = f.ms_learned;
            }
        }
    }
}

// Grid sizes of the persistent kernels from the launch config (0 = the
// occupancy maximum), clamped to what can be resident.
static void apply_launch(ve_ctx* c) {
    auto pick = [&](uint32_t want, int occ) { return int((want == 0 || int(want) > occ) ? occ : int(want)); };
    c->grid_trace = c->num_sms * pick(c->launch.trace_blocks_per_sm, c->occ_trace);
    c->grid_trace_count = c->num_sms * pick(c->launch.trace_blocks_per_sm, c->occ_trace_count);
    c->grid_shade = c->num_sms * pick(c->launch.shade_blocks_per_sm, c->occ_shade);
    // default: refill when 20 of 32 lanes are idle (measured on the depth-10
    // 1080p workload with the FLAT walk: 0.979 ms of trace per frame at 20
    // against 0.984 at 16 and 0.994 at 12; each refill is a dependent chain
    // of loads, and the cheaper the step, the fewer refills pay)
    if (c->launch.refill_threshold == 0 || c->launch.refill_threshold > 32) c->launch.refill_threshold = kDefaultRefill;
}

// Grid of a shading instance: the configured blocks per SM, capped at what
// that instance keeps resident (so the grid is one wave).
static uint32_t shade_grid(const ve_ctx* c, int mode, bool emit) {
    const int occ = emit ? c->occ_emit_mode[mode & 3] : c->occ_shade_mode[mode & 7];
    const int want = int(c->launch.shade_blocks_per_sm);
    return uint32_t(c->num_sms * ((want == 0 || want > occ) ? occ : want));
}

// Row ranges of a view: a split frame's band and, for its primary rays, the
// band widened by the rows the AvgPass reads around a pixel (the
// reconstruction radius, and 1 for the 4-neighbour filter).
static void set_rows(DevView& d, const ve_frame_config& f, bool split) {
    if (!split) {
        d.row_lo = 0; d.row_hi = f.height; d.g_lo = 0; d.g_hi = f.height;
        return;
    }
    const uint32_t halo = std::max<uint32_t>(f.reconstruction_radius, 1u);
    d.row_lo = f.row_begin;
    d.row_hi = f.row_end;
    d.g_lo = f.row_begin > halo ? f.row_begin - halo : 0u;
    d.g_hi = std::min<uint32_t>(f.row_end + halo, f.height);
}

// Path slots a view takes in a batch: spp per pixel (per pixel of the band
// for split frames), or the shade list's bound for scheduled frames.
static uint64_t view_paths(const ve_frame_config& f) {
    if (f.flags & VE_FRAME_SCHEDULED) return std::min<uint64_t>(f.shading_budget, 2ull * f.width * f.height);
    if (f.flags & VE_FRAME_SPLIT) {
        const uint32_t hi = std::min(f.row_end, f.height), lo = std::min(f.row_begin, hi);
        return uint64_t(hi - lo) * f.width * f.spp;
    }
    return uint64_t(f.width) * f.height * f.spp;
}

// The device view record of a view (everything but its offsets in the batch).
static void fill_view(DevView& d, const ve_view& v) {
    const ve_frame_config& f = v.frame;
    std::memset(&d, 0, sizeof(d));
    std::memcpy(d.cam, v.camera, sizeof(d.cam));
    d.scene = uint32_t(v.scene_id);
    d.W = f.width; d.H = f.height; d.spp = f.spp;
    d.bounces = f.bounces; d.cc_primary = f.primary_controlchecks; d.cc_bounce = f.bounce_controlchecks;
    d.recon_radius = f.reconstruction_radius; d.render_type = f.render_type; d.frame_index = f.frame_index;
    d.flags = f.flags;
    d.tiles_x = (f.width + 15) / 16;
    for (int k = 0; k < 3; k++) { d.sun[k] = f.sun_dir[k]; d.sky[k] = f.sky[k]; }
    d.sun_intensity = f.sun_intensity;
    d.decay = f.decay;
    d.variance_norm = f.variance_norm;
    d.w_pix = f.weight_pixels;
    d.w_var = f.weight_variance;
    d.pix_norm = f.pixels_norm;
    d.top_frac = f.top_fraction;
    d.mid_frac = f.mid_fraction;
    d.min_samples = std::min<uint32_t>(f.min_samples, 2u);
    d.budget = f.shading_budget;
    d.restir = f.restir;
    d.restir_m = f.restir_m;
    d.restir_nbrs = f.restir_spatial_neighbors;
    d.restir_max_m = f.restir_max_m;
    d.restir_radius = f.restir_spatial_radius;
    d.lb = LbParams{f.time, f.update_time, f.disable_stale_reset, f.sample_cap_direct, f.sample_cap_indirect,
                    f.firefly_k, f.firefly_floor};
    set_rows(d, f, (f.flags & VE_FRAME_SPLIT) != 0);
}

static int render_batch(ve_ctx* c, const ve_view* views, uint32_t nv, ve_frame_outputs* outs) {
    if (!c || !views || nv == 0) return fail(VE_ERR_INVALID, "render: no views");
    if (nv > 65535u) return fail(VE_ERR_INVALID, "render: at most 65535 views per batch");
    uint64_t pixels = 0, paths = 0;
    uint32_t tiles = 0, max_b = 0, min_b = ~0u, flags = 0;
    for (uint32_t i = 0; i < nv; i++) {
        const ve_view& v = views[i];
        const ve_frame_config& f = v.frame;
        min_b = std::min(min_b, f.bounces);
        if (v.scene_id < 0 || size_t(v.scene_id) >= c->scenes.size() || !c->scenes[v.scene_id].live)
            return fail(VE_ERR_NOT_FOUND, "render: unknown scene id " + std::to_string(v.scene_id));
        if (f.width == 0 || f.height == 0 || f.width > 16384 || f.height > 16384)
            return fail(VE_ERR_INVALID, "render: width/height must be in [1, 16384]");
        if (f.spp == 0 || f.spp > 1024) return fail(VE_ERR_INVALID, "render: spp must be in [1, 1024]");
        if (f.bounces + 2 > kMaxPasses) return fail(VE_ERR_INVALID, "render: bounces must be <= 16");
        if (f.render_type > VE_RENDER_VARIANCE) return fail(VE_ERR_INVALID, "render: unknown render type");
        // every DDA loop is bounded by its controlchecks; keep the bound finite
        if (f.primary_controlchecks > kMaxControlChecks || f.bounce_controlchecks > kMaxControlChecks)
            return fail(VE_ERR_INVALID, "render: controlchecks must be <= 65536");
        if (f.reconstruction_radius > 64) return fail(VE_ERR_INVALID, "render: reconstruction_radius must be <= 64");
        const uint32_t tx = (f.width + 15) / 16, ty = (f.height + 15) / 16;
        tiles += tx * ty;
        pixels += uint64_t(f.width) * f.height;
        paths += view_paths(f);
        max_b = std::max(max_b, f.bounces);
        flags |= f.flags;
    }
    if ((flags & VE_FRAME_SCHEDULED) && nv != 1)
        return fail(VE_ERR_INVALID, "render: VE_FRAME_SCHEDULED renders one view per call");
    if ((flags & VE_FRAME_SCHEDULED) && (flags & (VE_FRAME_LEARNED | VE_FRAME_TRAIN)))
        return fail(VE_ERR_INVALID, "render: VE_FRAME_SCHEDULED does not combine with the learned cache");
    if ((flags & VE_FRAME_EMISSIVE) && (flags & (VE_FRAME_LEARNED | VE_FRAME_TRAIN | VE_FRAME_TERMINATE_HASH)))
        return fail(VE_ERR_INVALID, "render: VE_FRAME_EMISSIVE does not combine with cache-terminated paths");
    if ((flags & VE_FRAME_LBUFFER) && nv != 1)
        return fail(VE_ERR_INVALID, "render: VE_FRAME_LBUFFER renders one view per call");
    if ((flags & VE_FRAME_LBUFFER) && (flags & (VE_FRAME_LEARNED | VE_FRAME_TRAIN | VE_FRAME_TERMINATE_HASH)))
        return fail(VE_ERR_INVALID, "render: VE_FRAME_LBUFFER does not combine with cache-terminated paths");
    for (uint32_t i = 0; i < nv; i++)
        if ((views[i].frame.flags & VE_FRAME_EMISSIVE) && views[i].frame.restir_m > 64)
            return fail(VE_ERR_INVALID, "render: restir_m must be <= 64");
    const bool split = (flags & VE_FRAME_SPLIT) != 0;
    if (!split) c->split_scene = -1;  // the GBuffer of a split frame is about to be overwritten
    if (split) {
        const ve_frame_config& f = views[0].frame;
        if (nv != 1) return fail(VE_ERR_INVALID, "render: VE_FRAME_SPLIT renders one view per call");
        if (flags & (VE_FRAME_SCHEDULED | VE_FRAME_EMISSIVE | VE_FRAME_LBUFFER | VE_FRAME_LEARNED | VE_FRAME_TRAIN |
                     VE_FRAME_TERMINATE_HASH))
            return fail(VE_ERR_INVALID, "render: VE_FRAME_SPLIT renders plain path-traced frames only");
        if (f.row_begin >= f.row_end || f.row_end > f.height)
            return fail(VE_ERR_INVALID, "render: VE_FRAME_SPLIT needs row_begin < row_end <= height");
        if (outs && (outs[0].rgb || outs[0].mapped || outs[0].mapped8 || outs[0].voxel_id || outs[0].hit_node))
            return fail(VE_ERR_INVALID, "render: a VE_FRAME_SPLIT frame's image comes from ve_split_resolve");
    }
    const bool async_out = (flags & VE_FRAME_ASYNC_OUTPUTS) != 0;
    if (async_out) {
        if (split) return fail(VE_ERR_INVALID, "render: VE_FRAME_SPLIT frames have no images to copy");
        for (uint32_t i = 0; outs && i < nv; i++)
            if (outs[i].gbuffer || outs[i].path_rgb)
                return fail(VE_ERR_INVALID,
                            "render: VE_FRAME_ASYNC_OUTPUTS copies voxel_id, hit_node, rgb, mapped and mapped8 only");
    }
    // path slots are 30 bits (queue entries carry two flag bits)
    if (paths >= (1ull << 30)) return fail(VE_ERR_CAPACITY, "render: more than 2^30 paths in one batch");
    // learned radiance cache: one per batch, attached to the views' scenes
    ve_nrc* nrc = nullptr;
    for (uint32_t i = 0; i < nv; i++) {
        if (!(views[i].frame.flags & (VE_FRAME_LEARNED | VE_FRAME_TRAIN))) continue;
        ve_nrc* m = c->scenes[views[i].scene_id].nrc;
        if (!m) return fail(VE_ERR_STATE, "render: VE_FRAME_LEARNED / VE_FRAME_TRAIN on a scene without a learned cache");
        if (nrc && m != nrc) return fail(VE_ERR_INVALID, "render: at most one learned cache per batch");
        nrc = m;
    }
    // VE_CFG_PIPELINE: plain frames whose primary pass takes no path to a
    // deposit (every view has a bounce) alternate between the two frame sets;
    // anything else runs on the main stream after the second set's frames
    const bool pipe = (c->cfg.flags & VE_CFG_PIPELINE) && !split && min_b >= 1 && !c->scenes_dirty &&
                      !(flags & (VE_FRAME_TIMING | VE_FRAME_COUNT_FETCH | VE_FRAME_PATH_RGB | VE_FRAME_LEARNED |
                                 VE_FRAME_TERMINATE_HASH | VE_FRAME_TRAIN | VE_FRAME_SCHEDULED | VE_FRAME_EMISSIVE |
                                 VE_FRAME_LBUFFER));
    if (!pipe) join_alt(c);
    const int set = pipe ? c->pipe_next : 0;
    if (pipe) {
        if (!c->alt.stream) {
            if (cudaStreamCreateWithFlags(&c->alt.stream, cudaStreamNonBlocking) != cudaSuccess ||
                cudaEventCreateWithFlags(&c->set_cache_done[0], cudaEventDisableTiming) != cudaSuccess ||
                cudaEventCreateWithFlags(&c->set_cache_done[1], cudaEventDisableTiming) != cudaSuccess ||
                cudaEventCreateWithFlags(&c->alt_done, cudaEventDisableTiming) != cudaSuccess ||
                cudaEventCreateWithFlags(&c->ops_ev, cudaEventDisableTiming) != cudaSuccess)
                return fail(VE_ERR_CUDA, "render: frame-set stream creation failed");
        }
        if (!c->alt.h_stats && cudaMallocHost(&c->alt.h_stats, ST_TOTAL * sizeof(unsigned long long)) != cudaSuccess)
            return fail(VE_ERR_NOMEM, "render: frame-set allocation failed");
        c->pipe_next ^= 1;
    }
    SetScope scope(c, set == 1);  // c->stream and the frame buffers are this set's from here on
    if (set == 1) {
        if (int e = c->counters.ensure(CNT_TOTAL)) return e;
        if (int e = c->stats.ensure(ST_TOTAL)) return e;
        if (c->ops_pending) {  // main-stream work since this set's last frame comes first
            VE_CUDA(cudaEventRecord(c->ops_ev, c->alt.stream));
            VE_CUDA(cudaStreamWaitEvent(c->stream, c->ops_ev, 0));
            c->ops_pending = false;
        }
    }
    int rc = ensure_frame(c, pixels, paths, nv);
    if (rc) return rc;
    int parity = 0;  // the device image set this frame's resolve writes
    if (async_out) {
        if (!c->copy_stream) {
            if (cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking) != cudaSuccess ||
                cudaEventCreateWithFlags(&c->frame_done, cudaEventDisableTiming) != cudaSuccess ||
                cudaEventCreateWithFlags(&c->copy_done[0], cudaEventDisableTiming) != cudaSuccess ||
                cudaEventCreateWithFlags(&c->copy_done[1], cudaEventDisableTiming) != cudaSuccess)
                return fail(VE_ERR_CUDA, "render: copy stream creation failed");
        }
        const void* before[] = {c->out_vid2.p, c->out_node2.p, c->out_rgb2.p, c->out_mapped2.p, c->out_m82.p};
        if (pixels > c->out_vid2.cap || 3 * pixels > c->out_rgb2.cap) cudaStreamSynchronize(c->copy_stream);
        if ((rc = c->out_vid2.ensure(pixels)) || (rc = c->out_node2.ensure(pixels)) ||
            (rc = c->out_rgb2.ensure(3 * pixels)) || (rc = c->out_mapped2.ensure(3 * pixels)) ||
            (rc = c->out_m82.ensure(pixels)))
            return rc;
        const void* after[] = {c->out_vid2.p, c->out_node2.p, c->out_rgb2.p, c->out_mapped2.p, c->out_m82.p};
        for (int i = 0; i < 5; i++)
            if (before[i] != after[i]) c->gen++;
        parity = c->out_parity;
    }
    const bool sched = (flags & VE_FRAME_SCHEDULED) != 0;
    uint32_t claim_size = 0;
    size_t scan_bytes = 0;
    if (sched) {
        SceneSlot& sc = c->scenes[views[0].scene_id];
        const void* before[] = {c->hitinfo.p, c->claim.p, c->sched_n.p, c->shade_list.p, c->scan_tmp.p, sc.rank};
        claim_size = 1024u;
        while (claim_size < 2ull * pixels) claim_size <<= 1;
        cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, c->sched_n.p, c->sched_n.p, int(pixels), c->stream);
        if ((rc = c->hitinfo.ensure(pixels)) || (rc = c->claim.ensure(3ull * claim_size)) ||
            (rc = c->sched_n.ensure(2 * pixels)) || (rc = c->shade_list.ensure(paths)) ||
            (rc = c->scan_tmp.ensure(scan_bytes)))
            return rc;
        if (!sc.rank) {
            if (cudaMalloc(&sc.rank, (2 + kRankBins) * 4) != cudaSuccess)
                return fail(VE_ERR_NOMEM, "render: scheduling state allocation failed");
            if ((rc = reset_rank(c, sc.rank))) return rc;
        }
        const void* after[] = {c->hitinfo.p, c->claim.p, c->sched_n.p, c->shade_list.p, c->scan_tmp.p, sc.rank};
        for (int i = 0; i < 6; i++)
            if (before[i] != after[i]) c->gen++;
    }
    if (nrc) {
        bool moved = false;
        if ((rc = nrc::prepare_frame(nrc, paths, &moved))) return rc;
        if (flags & VE_FRAME_TRAIN) {
            const void* old = c->p_aux.p;
            if ((rc = c->p_aux.ensure(paths))) return rc;
            moved |= old != c->p_aux.p;
        }
        if (moved) c->gen++;
    }
    if (flags & VE_FRAME_PATH_RGB) {
        const void* old = c->path_rgb.p;
        if ((rc = c->path_rgb.ensure(paths * 3))) return rc;
        if (old != c->path_rgb.p) c->gen++;
    }
    // emissive lights: the scenes' registries and reservoir tables, the
    // per-path NEE records and the registry commit's sort buffers
    // the trace's FLAT instance: every view's scene has a top table reaching
    // its leaves (depth 3..10)
    bool flat = true;
    for (uint32_t i = 0; i < nv; i++) {
        const SceneSlot& sc = c->scenes[views[i].scene_id];
        flat = flat && sc.top_level != 0u && sc.top_level == sc.depth;
    }
    std::vector<int> em_scenes;
    size_t em_sort_bytes = 0;
    if (flags & VE_FRAME_EMISSIVE) {
        for (uint32_t i = 0; i < nv; i++) {
            if (!(views[i].frame.flags & VE_FRAME_EMISSIVE)) continue;
            const int sc = views[i].scene_id;
            if (std::find(em_scenes.begin(), em_scenes.end(), sc) == em_scenes.end()) em_scenes.push_back(sc);
            if ((rc = ensure_emissive(c, c->scenes[sc]))) return rc;
        }
        constexpr int cap = 1 << kEmClaimLog2;
        cub::DeviceRadixSort::SortPairs(nullptr, em_sort_bytes, (const uint32_t*)nullptr, (uint32_t*)nullptr,
                                        (const uint32_t*)nullptr, (uint32_t*)nullptr, cap, 0, 32, c->stream);
        const void* before[] = {c->p_sdir.p, c->p_res.p, c->res_list.p, c->em_sort.p, c->em_sort_tmp.p};
        if ((rc = c->p_sdir.ensure(paths)) || (rc = c->p_res.ensure(paths)) || (rc = c->res_list.ensure(paths)) ||
            (rc = c->em_sort.ensure(4ull * cap)) || (rc = c->em_sort_tmp.ensure(em_sort_bytes)))
            return rc;
        const void* after[] = {c->p_sdir.p, c->p_res.p, c->res_list.p, c->em_sort.p, c->em_sort_tmp.p};
        for (int i = 0; i < 5; i++)
            if (before[i] != after[i]) c->gen++;
    }
    size_t lb_sort_bytes = 0;
    if (flags & VE_FRAME_LBUFFER) {
        if ((rc = ensure_lbuffer(c, c->scenes[views[0].scene_id]))) return rc;
        cub::DeviceRadixSort::SortPairs(nullptr, lb_sort_bytes, (const uint32_t*)nullptr, (uint32_t*)nullptr,
                                        (const uint32_t*)nullptr, (uint32_t*)nullptr, int(paths), 0, 15, c->stream);
        const void* before[] = {c->lb_rec.p, c->lb_keys.p, c->lb_idx.p, c->lb_tmp.p};
        const size_t idx_cap = c->lb_idx.cap;
        if ((rc = c->lb_rec.ensure(paths)) || (rc = c->lb_keys.ensure(2 * paths)) ||
            (rc = c->lb_idx.ensure(2 * paths + 2ull * kLbWidth)) || (rc = c->lb_tmp.ensure(lb_sort_bytes)))
            return rc;
        const void* after[] = {c->lb_rec.p, c->lb_keys.p, c->lb_idx.p, c->lb_tmp.p};
        for (int i = 0; i < 4; i++)
            if (before[i] != after[i]) c->gen++;
        if (before[2] != after[2] || idx_cap != c->lb_idx.cap || c->lb_iota < paths) {  // sort values: 0, 1, 2, ...
            k_iota<<<c->num_sms * 8, 256, 0, c->stream>>>(c->lb_idx.p, uint32_t(paths));
            c->lb_iota = paths;
        }
    }
    if ((rc = sync_scenes(c))) return rc;
    if (split) {  // the frame's deposits go to the per-frame table
        const int sid = views[0].scene_id;
        const void* before[] = {c->split_delta.p, c->d_scenes_split.p};
        if ((rc = c->split_delta.ensure(size_t(1) << c->cfg.hash_log2)) ||
            (rc = c->d_scenes_split.ensure(c->d_scenes.cap)) || (rc = c->split_cnt.ensure(2)))
            return rc;
        if (before[0] != c->split_delta.p || before[1] != c->d_scenes_split.p) {
            c->gen++;
            c->split_delta_clean = false;
        }
        if (!c->split_delta_clean)  // not exported since its last frame (or new): clear it
            VE_CUDA(cudaMemsetAsync(c->split_delta.p, 0, (size_t(1) << c->cfg.hash_log2) * sizeof(CacheEntry),
                                    c->stream));
        c->split_delta_clean = false;
        CacheEntry* delta = c->split_delta.p;
        VE_CUDA(cudaMemcpyAsync(c->d_scenes_split.p, c->d_scenes.p, c->scenes.size() * sizeof(DevScene),
                                cudaMemcpyDeviceToDevice, c->stream));
        VE_CUDA(cudaMemcpyAsync(&c->d_scenes_split.p[sid].cache, &delta, sizeof(delta), cudaMemcpyHostToDevice,
                                c->stream));
        VE_CUDA(cudaStreamSynchronize(c->stream));
        c->split_scene = sid;
        c->split_frame = views[0].frame;
    }
    // view table, written into a staging slot whose previous copy has run
    const int slot = c->staging_next;
    c->staging_next = (slot + 1) % ve_ctx::kStaging;
    VE_CUDA(cudaEventSynchronize(c->staging_ev[slot]));
    DevView* hv = c->h_views[slot];
    uint32_t tile_base = 0;
    uint64_t pix_base = 0, path_base = 0;
    for (uint32_t i = 0; i < nv; i++) {
        const ve_frame_config& f = views[i].frame;
        DevView& d = hv[i];
        fill_view(d, views[i]);
        d.pix_base = uint32_t(pix_base);
        d.tile_base = tile_base;
        // a split frame's paths are numbered from its band's first pixel: the
        // base wraps so that base + pixel * spp + sample is the slot (mod 2^64)
        d.path_base = (f.flags & VE_FRAME_SPLIT) ? path_base - uint64_t(f.row_begin) * f.width * f.spp : path_base;
        tile_base += d.tiles_x * ((f.height + 15) / 16);
        pix_base += uint64_t(f.width) * f.height;
        path_base += view_paths(f);
    }
    cudaStream_t st = c->stream;
    const bool timing = (flags & VE_FRAME_TIMING) != 0;
    const bool count = (flags & VE_FRAME_COUNT_FETCH) != 0;
    uint32_t launches = 0, trace_launches = 0;
    VE_CUDA(cudaMemcpyAsync(c->d_views.p, hv, sizeof(DevView) * nv, cudaMemcpyHostToDevice, st));
    VE_CUDA(cudaEventRecord(c->staging_ev[slot], st));
    uint64_t h2d = sizeof(DevView) * nv, d2h = 0;
    // events: 0 start, 1 after decay, 2 after primary, then per pass
    // (shade, trace) pairs, last = after resolve
    ve_ctx::TimingSlot* ts = nullptr;
    if (timing) {
        ts = &c->timing[c->timing_next];
        c->timing_next = (c->timing_next + 1) % ve_ctx::kTimingSlots;
        if (ts->pending) collect_timing(c, *ts, nullptr);
    }
    int ne = 0;
    auto rec = [&]() {
        if (timing) cudaEventRecord(ts->ev[ne], st);
        ne++;
    };
    // decay once per distinct scene (first view's decay factor)
    std::vector<std::pair<int, float>> decays;
    for (uint32_t i = 0; i < nv; i++) {
        const int sc = views[i].scene_id;
        bool seen = false;
        for (auto& d : decays) seen |= d.first == sc;
        // the lBuffer has no decay (its channels halve at their sample caps)
        if (!seen && !(views[i].frame.flags & VE_FRAME_LBUFFER)) decays.emplace_back(sc, views[i].frame.decay);
    }
    FrameArgs a{};
    a.views = c->d_views.p;
    a.n_views = nv;
    a.total_tiles = tiles;
    a.scenes = split ? c->d_scenes_split.p : c->d_scenes.p;
    a.mats = c->d_mats.p;
    a.p_ray_o = c->p_ray_o.p; a.p_ray_d = c->p_ray_d.p; a.p_tp = c->p_tp.p;
    a.p_direct = c->p_direct.p; a.p_indirect = c->p_indirect.p; a.p_pend = c->p_pend.p;
    a.p_hit = c->p_hit.p; a.p_meta = c->p_meta.p;
    a.live[0] = c->live0.p; a.live[1] = c->live1.p; a.rayq = c->rayq.p; a.rayq_sh = c->rayq.p + paths;
    a.counters = c->counters.p; a.stats = c->stats.p;
    a.gbuf = c->gbuf.p;
    a.out_vid = parity ? c->out_vid2.p : c->out_vid.p;
    a.out_node = parity ? c->out_node2.p : c->out_node.p;
    a.out_rgb = parity ? c->out_rgb2.p : c->out_rgb.p;
    a.out_mapped = parity ? c->out_mapped2.p : c->out_mapped.p;
    a.out_mapped8 = parity ? c->out_m82.p : c->out_m8.p;
    a.path_rgb = (flags & VE_FRAME_PATH_RGB) ? c->path_rgb.p : nullptr;
    a.refill = c->launch.refill_threshold;
    a.view_offset = 0;
    a.remaining = nullptr;
    const bool learned = nrc && (flags & VE_FRAME_LEARNED);
    const bool train = nrc && (flags & VE_FRAME_TRAIN);
    if (nrc) {
        a.nq = learned ? nrc->fq.p : nullptr;
        a.nstage = nrc->fstage.p;
        a.nq_cap = uint32_t(paths);
        a.ns = train ? nrc->fs.p : nullptr;
        a.nt = nrc->ftr.p;
        a.ns_cap = nrc->cfg.train_samples;
        // select ~1.25x the sample budget among the frame's paths (not every
        // path reaches a second vertex); the overflow stays plain
        const double frac = std::min(1.0, 1.25 * double(nrc->cfg.train_samples) / double(std::max<uint64_t>(paths, 1)));
        a.train_thresh = uint32_t(std::min(4294967295.0, frac * 4294967296.0));
        a.fallback_thr = nrc->cfg.fallback_threshold;
        a.val = nrc->val.p;
        a.val_mask = (1u << nrc::kValCellsLog2) - 1u;
        a.nrc_ready = nrc->trained_steps >= nrc::kReadySteps ? 1u : 0u;
        a.p_aux = train ? c->p_aux.p : nullptr;
    }
    if (sched) {
        a.hitinfo = c->hitinfo.p;
        a.claim_key = c->claim.p;
        a.claim_pix = c->claim.p + claim_size;
        a.claim_cnt = c->claim.p + 2ull * claim_size;
        a.claim_mask = claim_size - 1u;
        a.sched_n = c->sched_n.p;
        a.sched_off = c->sched_n.p + pixels;
        a.shade_list = c->shade_list.p;
        a.shade_cap = uint32_t(paths);
        a.rank = c->scenes[views[0].scene_id].rank;
    }
    if (flags & VE_FRAME_LBUFFER) {
        a.lb_rec = c->lb_rec.p;
        a.lb_key = c->lb_keys.p;
    }
    if (flags & VE_FRAME_EMISSIVE) {
        a.p_sdir = c->p_sdir.p;
        a.p_res = c->p_res.p;
        a.res_list = c->res_list.p;
    }
    const bool em = (flags & VE_FRAME_EMISSIVE) != 0;
    const bool lbm = (flags & VE_FRAME_LBUFFER) != 0;
    const bool nrcm = (flags & (VE_FRAME_LEARNED | VE_FRAME_TERMINATE_HASH | VE_FRAME_TRAIN)) != 0;
    const int mode = (em ? kModeEm : 0) | (lbm ? kModeLb : 0) | (nrcm ? kModeNrc : 0);
    // the frame's kernel sequence (no host synchronisation inside)
    // part 0: the whole frame; a pipelined frame runs as part 1 (primary and
    // trace pass 0, which read no radiance cache) and part 2 (the decay and
    // everything after), with the wait for the other set's cache work between
    auto decay = [&]() {
        for (auto& d : decays) {
            if (d.second != 1.0f) {
                const uint32_t n = 1u << c->cfg.hash_log2;
                k_decay<<<c->num_sms * 8, 256, 0, st>>>(c->scenes[d.first].cache, n, d.second);
                launches++;
            }
        }
    };
    auto enqueue = [&](int part) {
        const bool head = part != 2, tail = part != 1;
        if (head) {
        cudaMemsetAsync(c->counters.p, 0, CNT_TOTAL * sizeof(uint32_t), st);
        cudaMemsetAsync(c->stats.p, 0, ST_TOTAL * sizeof(unsigned long long), st);
        // paths of pixels without a primary hit are never spawned: their
        // debug slots read as zero
        if (flags & VE_FRAME_PATH_RGB) cudaMemsetAsync(c->path_rgb.p, 0, paths * 3 * sizeof(float), st);
        // lBuffer frames: row 0 (no deposit) for paths that are never spawned
        if (lbm) cudaMemsetAsync(c->lb_keys.p, 0, paths * sizeof(uint32_t), st);
        rec();
        if (part == 0) decay();
        rec();
        if (count) launch_primary<true>(mode, tiles, st, a);
        else launch_primary<false>(mode, tiles, st, a);
        launches++;
        if (sched) {  // schedule -> rank -> shade list -> thresholds -> emit
            cudaMemsetAsync(a.claim_key, 0, 4ull * claim_size, st);
            cudaMemsetAsync(a.claim_pix, 0xFF, 4ull * claim_size, st);
            cudaMemsetAsync(a.claim_cnt, 0, 4ull * claim_size, st);
            cudaMemsetAsync(a.rank + 2, 0, 4ull * kRankBins, st);
            const int g = c->num_sms * 8;
            k_sched_claim<<<g, 256, 0, st>>>(a);
            k_sched_rank<<<g, 256, 0, st>>>(a);
            size_t b = scan_bytes;
            cub::DeviceScan::ExclusiveSum(c->scan_tmp.p, b, a.sched_n, a.sched_off, int(pixels), st);
            k_sched_list<<<g, 256, 0, st>>>(a);
            k_sched_threshold<<<1, 1, 0, st>>>(a.rank, a.views);
            launch_sched_emit(mode, shade_grid(c, mode & ~kModeNrc, true), st, a);
            launches += 6;
        }
        rec();
        }
        if (part == 2) decay();
        for (uint32_t pass = head ? 0u : 1u; pass <= (tail ? max_b + 1u : 0u); pass++) {
            if (pass > 0) {  // pass 0 runs inside the fused primary
                launch_shade(mode, shade_grid(c, mode, false), st, a, pass);
                launches++;
            }
            rec();
            if (pass <= max_b) {
                if (em) {
                    if (count) k_trace<true, true><<<c->grid_trace_count, 256, 0, st>>>(a, pass);
                    else k_trace<false, true><<<c->grid_trace, 256, 0, st>>>(a, pass);
                } else {
                    if (count) k_trace<true><<<c->grid_trace_count, 256, 0, st>>>(a, pass);
                    else if (flat) k_trace<false, false, true><<<c->grid_trace, 256, 0, st>>>(a, pass);
                    else k_trace<false><<<c->grid_trace, 256, 0, st>>>(a, pass);
                }
                launches++;
                trace_launches++;
            }
            rec();
        }
        if (!tail) return;
        if (learned || train) {
            if (learned) {
                nrc::launch_infer(nrc, st, nrc::infer_args(nrc, nrc->fq.p, c->counters.p + CNT_NRC_Q, a.nq_cap),
                                  nrc->fx.p, StagePath{a}, ApplyDeposit{a});
                launches += 2;
            }
            if (train) {
                nrc::enqueue_zero_grads(nrc, st);
                nrc::launch_train(nrc, st, nrc->fs.p, nrc->ftr.p, c->counters.p + CNT_NRC_S, a.ns_cap,
                                  1.0f / (3.0f * float(a.ns_cap)));
                nrc::launch_adam(nrc, st);
                launches += 4;
            }
            rec();
        }
        if (lbm) {  // AccumPass: the frame's deposits into the lBuffer, row by row
            const uint32_t capn = uint32_t(paths);
            uint32_t* kin = c->lb_keys.p;
            uint32_t* kout = kin + capn;
            uint32_t* vin = c->lb_idx.p;
            uint32_t* vout = vin + capn;
            uint32_t* rs = vout + capn;
            uint32_t* re = rs + kLbWidth;
            cudaMemsetAsync(rs, 0, 2ull * kLbWidth * sizeof(uint32_t), st);
            size_t b = lb_sort_bytes;
            cub::DeviceRadixSort::SortPairs(c->lb_tmp.p, b, kin, kout, vin, vout, int(capn), 0, 15, st);
            k_lb_bounds<<<c->num_sms * 8, 256, 0, st>>>(kout, capn, rs, re);
            k_lb_apply<<<kLbWidth / 8, 256, 0, st>>>(a.scenes, a.views, c->lb_rec.p, vout, rs, re);
            launches += 3;
        }
        if (split) {
            // the AvgPass follows the merge (ve_split_resolve)
        } else if (lbm) {
            k_resolve<true><<<tiles, 256, 0, st>>>(a);
            launches++;
        } else {
            k_resolve<<<tiles, 256, 0, st>>>(a);
            launches++;
        }
        if (flags & VE_FRAME_EMISSIVE) {  // this frame's lights and reservoirs, for the next frame
            constexpr int cap = 1 << kEmClaimLog2;
            uint32_t* kin = c->em_sort.p;
            uint32_t* kout = kin + cap;
            uint32_t* vin = kin + 2 * cap;
            uint32_t* vout = kin + 3 * cap;
            for (int sc : em_scenes) {
                k_em_keys<<<c->num_sms * 4, 256, 0, st>>>(a.scenes, uint32_t(sc), kin, vin);
                size_t b = em_sort_bytes;
                cub::DeviceRadixSort::SortPairs(c->em_sort_tmp.p, b, kin, kout, vin, vout, cap, 0, 32, st);
                k_em_append<<<1, 1024, 0, st>>>(a.scenes, uint32_t(sc), vout, c->stats.p);
                launches += 3;
            }
            k_res_commit<<<c->num_sms * 4, 256, 0, st>>>(a);
            launches++;
        }
        rec();
        k_accum_stats<<<1, 32, 0, st>>>(c->stats.p, c->totals.p);
        launches++;
    };
    // this frame's resolve overwrites an image set whose copy may be pending
    if (c->copy_stream) VE_CUDA(cudaStreamWaitEvent(st, c->copy_done[parity], 0));
    const bool use_graph = !timing && !(c->cfg.flags & VE_CFG_NO_GRAPHS);
    // one part of the frame: enqueued directly, or as the replay of its
    // cached CUDA graph (captured on first use)
    auto run = [&](int part) -> int {
        if (!use_graph) {
            enqueue(part);
            return VE_OK;
        }
        std::vector<uint64_t> key = {c->gen, nv, tiles, max_b,
                                     flags & (VE_FRAME_COUNT_FETCH | VE_FRAME_PATH_RGB | VE_FRAME_LEARNED |
                                              VE_FRAME_TERMINATE_HASH | VE_FRAME_TRAIN | VE_FRAME_SCHEDULED |
                                              VE_FRAME_EMISSIVE | VE_FRAME_LBUFFER | VE_FRAME_SPLIT),
                                     paths, uint64_t(c->grid_trace), uint64_t(c->grid_shade),
                                     uint64_t(c->launch.refill_threshold), uint64_t(uintptr_t(nrc)),
                                     uint64_t(a.nrc_ready)};
        for (auto& d : decays) {
            uint32_t bits;
            std::memcpy(&bits, &d.second, 4);
            key.push_back((uint64_t(uint32_t(d.first)) << 32) | bits);
        }
        for (int sc : em_scenes) key.push_back((1ull << 62) | uint64_t(uint32_t(sc)));
        key.push_back((1ull << 61) | uint64_t(parity));
        key.push_back((1ull << 59) | uint64_t(flat));
        key.push_back((1ull << 60) | (uint64_t(set) << 8) | uint64_t(part));
        ve_ctx::GraphEntry* ge = nullptr;
        for (auto& g : c->graphs)
            if (g.key == key) ge = &g;
        if (!ge) {
            const uint32_t l0 = launches, t0 = trace_launches;
            cudaGraph_t graph = nullptr;
            VE_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            enqueue(part);
            const cudaError_t ce = cudaStreamEndCapture(st, &graph);
            if (ce != cudaSuccess) return fail(VE_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
            cudaGraphExec_t exec = nullptr;
            const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
            cudaGraphDestroy(graph);
            if (ie != cudaSuccess) return fail(VE_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie));
            if (c->graphs.size() >= 16) {
                auto oldest = std::min_element(c->graphs.begin(), c->graphs.end(),
                                               [](const auto& x, const auto& y) { return x.last_use < y.last_use; });
                cudaGraphExecDestroy(oldest->exec);
                c->graphs.erase(oldest);
            }
            ve_ctx::GraphEntry e;
            e.key = key;
            e.exec = exec;
            e.launches = launches - l0;
            e.trace_launches = trace_launches - t0;
            c->graphs.push_back(e);
            ge = &c->graphs.back();
            c->graph_captures++;
        } else {
            launches += ge->launches;
            trace_launches += ge->trace_launches;
            c->graph_replays++;
        }
        ge->last_use = ++c->graph_clock;
        VE_CUDA(cudaGraphLaunch(ge->exec, st));
        return VE_OK;
    };
    if (!pipe) {
        if ((rc = run(0))) return rc;
    } else {
        if ((rc = run(1))) return rc;
        // the other set's frame: its deposits and AvgPass before this decay
        VE_CUDA(cudaStreamWaitEvent(st, c->set_cache_done[set ^ 1], 0));
        if ((rc = run(2))) return rc;
        VE_CUDA(cudaEventRecord(c->set_cache_done[set], st));
    }
    VE_CUDA(cudaGetLastError());
    c->last_launches = launches;
    c->last_trace_launches = trace_launches;
    c->last_timing = timing;
    std::memset(&c->last, 0, sizeof(c->last));
    if (timing) {
        ts->n = ne;
        ts->passes = max_b + 2u;
        ts->learned = learned || train;
        ts->pending = true;
        c->last_timing_slot = int(ts - c->timing);
    } else {
        c->last_timing_slot = -1;
    }
    VE_CUDA(cudaMemcpyAsync(c->h_stats, c->stats.p, ST_TOTAL * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    // host outputs
    if (outs && async_out) {  // on the copy stream, after the frame; the call does not wait
        VE_CUDA(cudaEventRecord(c->frame_done, st));
        VE_CUDA(cudaStreamWaitEvent(c->copy_stream, c->frame_done, 0));
        cudaStream_t cs = c->copy_stream;
        uint64_t pb = 0;
        for (uint32_t i = 0; i < nv; i++) {
            const ve_frame_config& f = views[i].frame;
            const uint64_t np = uint64_t(f.width) * f.height;
            const ve_frame_outputs& o = outs[i];
            if (o.voxel_id) { VE_CUDA(cudaMemcpyAsync(o.voxel_id, a.out_vid + pb, np * 4, cudaMemcpyDeviceToHost, cs)); d2h += np * 4; }
            if (o.hit_node) { VE_CUDA(cudaMemcpyAsync(o.hit_node, a.out_node + pb, np * 4, cudaMemcpyDeviceToHost, cs)); d2h += np * 4; }
            if (o.rgb) { VE_CUDA(cudaMemcpyAsync(o.rgb, a.out_rgb + 3 * pb, np * 12, cudaMemcpyDeviceToHost, cs)); d2h += np * 12; }
            if (o.mapped) { VE_CUDA(cudaMemcpyAsync(o.mapped, a.out_mapped + 3 * pb, np * 12, cudaMemcpyDeviceToHost, cs)); d2h += np * 12; }
            if (o.mapped8) { VE_CUDA(cudaMemcpyAsync(o.mapped8, a.out_mapped8 + pb, np * 4, cudaMemcpyDeviceToHost, cs)); d2h += np * 4; }
            pb += np;
        }
        VE_CUDA(cudaEventRecord(c->copy_done[parity], cs));
        c->out_parity = parity ^ 1;
    } else if (outs) {
        uint64_t pb = 0, qb = 0;
        for (uint32_t i = 0; i < nv; i++) {
            const ve_frame_config& f = views[i].frame;
            const uint64_t np = uint64_t(f.width) * f.height;
            const uint64_t nq = view_paths(f);
            ve_frame_outputs& o = outs[i];
            if (split) {  // the band's rows
                const uint64_t r0 = uint64_t(f.row_begin) * f.width, nr = uint64_t(f.row_end - f.row_begin) * f.width;
                if (o.gbuffer) {
                    VE_CUDA(cudaMemcpyAsync(o.gbuffer + 4 * r0, c->gbuf.p + pb + r0, nr * 16, cudaMemcpyDeviceToHost, st));
                    d2h += nr * 16;
                }
                if (o.path_rgb && (f.flags & VE_FRAME_PATH_RGB)) {
                    VE_CUDA(cudaMemcpyAsync(o.path_rgb + 3 * r0 * f.spp, c->path_rgb.p + 3 * qb, nr * f.spp * 12,
                                            cudaMemcpyDeviceToHost, st));
                    d2h += nr * f.spp * 12;
                }
                continue;
            }
            if (o.gbuffer) { VE_CUDA(cudaMemcpyAsync(o.gbuffer, c->gbuf.p + pb, np * 16, cudaMemcpyDeviceToHost, st)); d2h += np * 16; }
            if (o.voxel_id) { VE_CUDA(cudaMemcpyAsync(o.voxel_id, c->out_vid.p + pb, np * 4, cudaMemcpyDeviceToHost, st)); d2h += np * 4; }
            if (o.hit_node) { VE_CUDA(cudaMemcpyAsync(o.hit_node, c->out_node.p + pb, np * 4, cudaMemcpyDeviceToHost, st)); d2h += np * 4; }
            if (o.rgb) { VE_CUDA(cudaMemcpyAsync(o.rgb, c->out_rgb.p + 3 * pb, np * 12, cudaMemcpyDeviceToHost, st)); d2h += np * 12; }
            if (o.mapped) { VE_CUDA(cudaMemcpyAsync(o.mapped, c->out_mapped.p + 3 * pb, np * 12, cudaMemcpyDeviceToHost, st)); d2h += np * 12; }
            if (o.mapped8) { VE_CUDA(cudaMemcpyAsync(o.mapped8, c->out_m8.p + pb, np * 4, cudaMemcpyDeviceToHost, st)); d2h += np * 4; }
            if (o.path_rgb && (f.flags & VE_FRAME_PATH_RGB)) {
                VE_CUDA(cudaMemcpyAsync(o.path_rgb, c->path_rgb.p + 3 * qb, nq * 12, cudaMemcpyDeviceToHost, st));
                d2h += nq * 12;
            }
            pb += np;
            qb += nq;
        }
        VE_CUDA(cudaStreamSynchronize(st));
    }
    if (set == 1) {
        VE_CUDA(cudaEventRecord(c->alt_done, st));
        c->alt_busy = true;
    }
    c->last_set = set;
    c->last_h2d = h2d;
    c->last_d2h = d2h;
    c->tot_frames++;
    c->tot_h2d += h2d;
    c->tot_d2h += d2h;
    c->tot_launches += launches;
    c->tot_trace_launches += trace_launches;
    if (train) nrc->trained_steps++;
    return VE_OK;
}

// Batch of independent rays through the device DDA (the same raycast the
// frame kernels run): 8 words per ray {status, hit node, material, x, y, z,
// size, checks} as Raycast / RaycastCounted (internal.glsl:297-400) reports
// them.  VE_RAYCAST_FULL_WALK descends every level per step (the
// fetch-counting variant) instead of starting from the top table.
template <bool FULL>
__global__ void __launch_bounds__(256) k_raycast_batch(DevScene S, const float* __restrict__ in, uint64_t n,
                                                       uint32_t cc, uint32_t* __restrict__ out) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        const f3 o = mk(in[3 * i + 0], in[3 * i + 1], in[3 * i + 2]);
        const f3 d = mk(in[3 * (n + i) + 0], in[3 * (n + i) + 1], in[3 * (n + i) + 2]);
        RayCount rc;
        const Hit h = raycast<FULL>(S.nodes, S.n_words, S.depth, S.top, S.top_level, o, d, cc, rc);
        uint32_t* w = out + 8 * i;
        w[0] = h.status; w[1] = h.id; w[2] = h.material;
        w[3] = h.x; w[4] = h.y; w[5] = h.z;
        w[6] = h.size; w[7] = h.checks;
    }
}

// Split frames: the per-frame deposit table as records {vid, count, luma^2,
// r, g, b, weight, 0}, compacted by a warp-aggregated counter; the entries
// read are cleared, so the table is empty for the next split frame.
__global__ void __launch_bounds__(256) k_split_export(CacheEntry* __restrict__ t, uint32_t n,
                                                      uint4* __restrict__ out, uint32_t cap, uint32_t* cnt) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += stride) {  // uniform per warp
        const uint32_t i = base + threadIdx.x;
        CacheEntry e{};
        if (i < n) e = t[i];
        const bool live = i < n && e.key != 0u;
        if (live) t[i] = CacheEntry{};
        const uint32_t j = warp_append(live, cnt);
        if (live && j < cap) {
            out[2ull * j + 0] = make_uint4(e.key, e.count, __float_as_uint(e.l2), __float_as_uint(e.rgbw.x));
            out[2ull * j + 1] = make_uint4(__float_as_uint(e.rgbw.y), __float_as_uint(e.rgbw.z),
                                           __float_as_uint(e.rgbw.w), 0u);
        }
    }
}

// Adds one rank's records into the cache.  A part holds each voxel once
// (it comes from one deposit table), so every entry sees one addition per
// part and the parts' launch order fixes the order of its sums.
__global__ void __launch_bounds__(256) k_split_merge(CacheEntry* cache, uint32_t log2n, uint32_t probes,
                                                     const uint4* __restrict__ rec, uint32_t n, uint32_t* dropped) {
    uint32_t drops = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint4 a = rec[2ull * i + 0], b = rec[2ull * i + 1];
        if (a.x == 0u || a.y == 0u) continue;
        const int s = cache_claim(cache, log2n, probes, a.x);
        if (s < 0) {
            drops++;
            continue;
        }
        CacheEntry* e = cache + s;
        atomicAdd(&e->count, a.y);
        atomicAdd(&e->l2, __uint_as_float(a.z));
        atomicAdd(&e->rgbw, make_float4(__uint_as_float(a.w), __uint_as_float(b.x), __uint_as_float(b.y),
                                        __uint_as_float(b.z)));
    }
    if (drops) atomicAdd(dropped, drops);
}

}  // namespace ve

// ===========================================================================
// C ABI
// ===========================================================================
using namespace ve;

extern "C" {

const char* ve_last_error(void) { return g_err.c_str(); }

int ve_ctx_create(const ve_renderer_config* cfg, ve_ctx** out) {
    if (!out) return fail(VE_ERR_INVALID, "ctx_create: null output");
    *out = nullptr;
    ve_renderer_config c{};
    c.device = 0;
    c.hash_log2 = 22;
    c.hash_probes = 64;
    if (cfg) c = *cfg;
    if (c.hash_log2 < 8 || c.hash_log2 > 28) return fail(VE_ERR_INVALID, "ctx_create: hash_log2 must be in [8, 28]");
    if (c.hash_probes == 0) c.hash_probes = 64;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(VE_ERR_CUDA, "ctx_create: no CUDA device available");
    if (c.device < 0 || c.device >= ndev) return fail(VE_ERR_INVALID, "ctx_create: bad device index");
    VE_CUDA(cudaSetDevice(c.device));
    ve_ctx* x = new ve_ctx();
    x->device = c.device;
    x->cfg = c;
    cudaDeviceGetAttribute(&x->num_sms, cudaDevAttrMultiProcessorCount, c.device);
    if (cudaStreamCreateWithFlags(&x->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete x;
        return fail(VE_ERR_CUDA, "ctx_create: stream creation failed");
    }
    for (auto& slot : x->timing)
        for (auto& e : slot.ev) cudaEventCreate(&e);
    {
        // scale factors of the Halton digit loop: f_0 = 1/b, f_{k+1} = f_k / b,
        // the same IEEE single-precision division sequence as the loop itself
        static const uint32_t bases[16] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53};
        float tab[16][24];
        for (int r = 0; r < 16; r++) {
            volatile float f = 1.0f;
            for (int k = 0; k < 24; k++) {
                f = f / float(bases[r]);
                tab[r][k] = f;
            }
        }
        // shading normals of the 19^3 stored gradients: normalize, 10-10-10
        // code of packNormalAccum, UnpackNormal, normalize (host IEEE single)
        static float4 ntab[19 * 19 * 19];
        for (int ix = -9; ix <= 9; ix++)
            for (int iy = -9; iy <= 9; iy++)
                for (int iz = -9; iz <= 9; iz++) {
                    volatile float ax = float(ix), ay = float(iy), az = float(iz);
                    const float len = std::sqrt((ax * ax + ay * ay) + az * az);
                    float n[3];
                    if (len > 0.001f) { n[0] = ax / len; n[1] = ay / len; n[2] = az / len; }
                    else { n[0] = 0.0f; n[1] = 1.0f; n[2] = 0.0f; }
                    float u[3];
                    for (int c = 0; c < 3; c++) {
                        int q = int(std::round((n[c] + 1.0f) * 511.0f));
                        q = q < 0 ? 0 : (q > 1022 ? 1022 : q);
                        u[c] = float(uint32_t(q)) / 511.0f - 1.0f;
                    }
                    const float s2 = std::sqrt((u[0] * u[0] + u[1] * u[1]) + u[2] * u[2]);
                    ntab[((ix + 9) * 19 + (iy + 9)) * 19 + (iz + 9)] = make_float4(u[0] / s2, u[1] / s2, u[2] / s2, 0.0f);
                }
        // through the context's non-blocking stream, waited for before the
        // host tables go out of scope and before any kernel reads them
        if (cudaMemcpyToSymbolAsync(g_normal_table, ntab, sizeof(ntab), 0, cudaMemcpyHostToDevice, x->stream) !=
                cudaSuccess ||
            cudaMemcpyToSymbolAsync(c_halton_f, tab, sizeof(tab), 0, cudaMemcpyHostToDevice, x->stream) != cudaSuccess ||
            cudaStreamSynchronize(x->stream) != cudaSuccess) {
            cudaStreamDestroy(x->stream);
            delete x;
            return fail(VE_ERR_CUDA, "ctx_create: constant table upload failed");
        }
    }
    int bt = 0, btc = 0, bs = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bt, k_trace<false>, 256, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&btc, k_trace<true>, 256, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bs, k_shade<0>, 256, 0);
    x->occ_trace = std::max(bt, 1);
    x->occ_trace_count = std::max(btc, 1);
    x->occ_shade = std::max(bs, 1);
    {
        int o[8] = {0};
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o[0], k_shade<0>, 256, 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o[kModeEm], k_shade<kModeEm>, 256, 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o[kModeLb], k_shade<kModeLb>, 256, 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o[kModeEm | kModeLb], k_shade<kModeEm | kModeLb>, 256, 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o[kModeNrc], k_shade<kModeNrc>, 256, 0);
        for (int m = 0; m < 8; m++) x->occ_shade_mode[m] = std::max(o[m], 1);
        int e[4] = {0};
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&e[0], k_sched_emit<0>, 256, 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&e[kModeEm], k_sched_emit<kModeEm>, 256, 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&e[kModeLb], k_sched_emit<kModeLb>, 256, 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&e[kModeEm | kModeLb], k_sched_emit<kModeEm | kModeLb>, 256,
                                                      0);
        for (int m = 0; m < 4; m++) x->occ_emit_mode[m] = std::max(e[m], 1);
    }
    apply_launch(x);
    int rc = 0;
    for (auto& e : x->staging_ev) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    if ((rc = x->counters.ensure(CNT_TOTAL)) || (rc = x->stats.ensure(ST_TOTAL)) ||
        (rc = x->totals.ensure(ST_TOTAL)) || (rc = x->d_mats.ensure(128))) {
        ve_ctx_destroy(x);
        return rc;
    }
    cudaMallocHost(&x->h_stats, ST_TOTAL * sizeof(unsigned long long));
    // on the context's non-blocking stream, finished before the first use
    cudaMemsetAsync(x->d_mats.p, 0, 128 * sizeof(DevMaterial), x->stream);
    cudaMemsetAsync(x->totals.p, 0, ST_TOTAL * sizeof(unsigned long long), x->stream);
    cudaMemsetAsync(x->stats.p, 0, ST_TOTAL * sizeof(unsigned long long), x->stream);
    if (cudaStreamSynchronize(x->stream) != cudaSuccess) {
        ve_ctx_destroy(x);
        return fail(VE_ERR_CUDA, "ctx_create: initialisation failed");
    }
    *out = x;
    return VE_OK;
}

int ve_ctx_destroy(ve_ctx* c) {
    if (!c) return VE_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    while (!c->nrcs.empty()) ve_nrc_destroy(c->nrcs.back());
    for (auto& s : c->scenes) {
        if (s.alloc) cudaFree(s.alloc);
        if (s.cache) cudaFree(s.cache);
        if (s.top) cudaFree(s.top);
        if (s.rank) cudaFree(s.rank);
        if (s.lbuf) cudaFree(s.lbuf);
        if (s.ntab) cudaFree(s.ntab);
        free_emissive(s);
    }
    c->d_scenes.release(); c->d_mats.release(); c->d_views.release();
    c->p_ray_o.release(); c->p_ray_d.release(); c->p_tp.release(); c->p_direct.release();
    c->p_indirect.release(); c->p_pend.release(); c->p_hit.release(); c->p_meta.release();
    c->live0.release(); c->live1.release(); c->rayq.release(); c->counters.release(); c->stats.release();
    c->p_aux.release();
    c->hitinfo.release(); c->claim.release(); c->sched_n.release(); c->shade_list.release(); c->scan_tmp.release();
    c->gbuf.release(); c->out_vid.release(); c->out_node.release(); c->out_rgb.release();
    c->out_mapped.release(); c->out_m8.release(); c->path_rgb.release(); c->ray_in.release(); c->ray_out.release();
    c->p_sdir.release(); c->p_res.release(); c->res_list.release(); c->em_sort.release(); c->em_sort_tmp.release();
    c->lb_rec.release(); c->lb_keys.release(); c->lb_idx.release(); c->lb_tmp.release();
    c->split_delta.release(); c->d_scenes_split.release(); c->split_cnt.release();
    if (c->copy_stream) {
        cudaStreamSynchronize(c->copy_stream);
        cudaStreamDestroy(c->copy_stream);
    }
    if (c->frame_done) cudaEventDestroy(c->frame_done);
    for (auto& e : c->copy_done)
        if (e) cudaEventDestroy(e);
    c->out_vid2.release(); c->out_node2.release(); c->out_rgb2.release(); c->out_mapped2.release();
    c->out_m82.release();
    for (int k = 0; k < ve_ctx::kStaging; k++) {
        if (c->h_views[k]) cudaFreeHost(c->h_views[k]);
        if (c->staging_ev[k]) cudaEventDestroy(c->staging_ev[k]);
    }
    c->totals.release();
    if (c->h_stats) cudaFreeHost(c->h_stats);
    {
        FrameSet& a = c->alt;
        if (a.stream) {
            cudaStreamSynchronize(a.stream);
            cudaStreamDestroy(a.stream);
        }
        a.d_views.release(); a.p_ray_o.release(); a.p_ray_d.release(); a.p_tp.release(); a.p_direct.release();
        a.p_indirect.release(); a.p_pend.release(); a.p_hit.release(); a.p_meta.release(); a.gbuf.release();
        a.live0.release(); a.live1.release(); a.rayq.release(); a.counters.release(); a.stats.release();
        if (a.h_stats) cudaFreeHost(a.h_stats);
        for (auto& e : c->set_cache_done)
            if (e) cudaEventDestroy(e);
        if (c->alt_done) cudaEventDestroy(c->alt_done);
        if (c->ops_ev) cudaEventDestroy(c->ops_ev);
    }
    for (auto& slot : c->timing)
        for (auto& e : slot.ev)
            if (e) cudaEventDestroy(e);
    for (auto& g : c->graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return VE_OK;
}

int ve_ctx_stream(ve_ctx* c, void** stream) {
    if (!c || !stream) return fail(VE_ERR_INVALID, "ctx_stream: null argument");
    *stream = c->stream;
    return VE_OK;
}

int ve_ctx_join(ve_ctx* c) {
    if (!c) return fail(VE_ERR_INVALID, "ctx_join: null context");
    if (c->alt_busy) VE_CUDA(cudaStreamWaitEvent(c->stream, c->alt_done, 0));
    c->alt_busy = false;
    return VE_OK;
}

int ve_ctx_synchronize(ve_ctx* c) {
    if (!c) return fail(VE_ERR_INVALID, "ctx_synchronize: null context");
    VE_CUDA(cudaStreamSynchronize(c->stream));
    if (c->alt.stream) VE_CUDA(cudaStreamSynchronize(c->alt.stream));
    if (c->copy_stream) VE_CUDA(cudaStreamSynchronize(c->copy_stream));
    return VE_OK;
}

}  // extern "C"

namespace ve {

// Device scratch of the bulk builder, freed on every exit path.
struct BuildScratch {
    std::vector<void*> ptrs;
    ~BuildScratch() {
        for (void* p : ptrs) cudaFree(p);
    }
    template <typename T>
    T* alloc(size_t n) {
        void* p = nullptr;
        if (cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) return nullptr;
        ptrs.push_back(p);
        return static_cast<T*>(p);
    }
};

#define VE_BUILD_ALLOC(ptr, T, n)                                    \
    T* ptr = scratch.alloc<T>(n);                                   \
    if (!ptr) return fail(VE_ERR_NOMEM, "scene_build: device allocation failed")

// Node words of OctreeCPU::insert (all voxels) + Octree::set, built on the
// device (builder.cuh).  `xyzm` is a device array of n (x, y, z, material).
// On success *words is a cudaMalloc'd array of *n_words words placed 7 words
// into the allocation (*alloc), like an uploaded scene.
static int build_scene_words(ve_ctx* c, const uint32_t* xyzm, uint64_t n, uint32_t D, void** alloc,
                             uint32_t** words, uint64_t* n_words) {
    using namespace build;
    cudaStream_t st = c->stream;
    BuildScratch scratch;
    const int grid = c->num_sms * 8;
    auto run_cub = [&](auto&& fn) -> int {  // size query, then the run
        size_t bytes = 0;
        if (fn(nullptr, bytes) != cudaSuccess) return fail(VE_ERR_CUDA, "scene_build: cub size query failed");
        void* tmp = scratch.alloc<uint8_t>(bytes);
        if (!tmp) return fail(VE_ERR_NOMEM, "scene_build: device allocation failed");
        if (fn(tmp, bytes) != cudaSuccess) return fail(VE_ERR_CUDA, "scene_build: cub call failed");
        return VE_OK;
    };
    auto empty_scene = [&]() -> int {  // no voxel: OctreeCPU has no root, Octree::set keeps 8 zero words
        void* a = nullptr;
        if (cudaMalloc(&a, 16 * 4) != cudaSuccess) return fail(VE_ERR_NOMEM, "scene_build: allocation failed");
        VE_CUDA(cudaMemsetAsync(a, 0, 16 * 4, st));
        VE_CUDA(cudaStreamSynchronize(st));
        *alloc = a;
        *words = reinterpret_cast<uint32_t*>(a) + 7;
        *n_words = 8;
        return VE_OK;
    };
    if (n == 0) return empty_scene();
    int rc;
    // 1. keys, stable sort, last voxel per position
    VE_BUILD_ALLOC(keys, uint64_t, n);
    VE_BUILD_ALLOC(keys_s, uint64_t, n);
    VE_BUILD_ALLOC(idx, uint32_t, n);
    VE_BUILD_ALLOC(idx_s, uint32_t, n);
    VE_BUILD_ALLOC(flag, uint8_t, n);
    VE_BUILD_ALLOC(nsel, uint64_t, 1);
    k_keys<<<grid, 256, 0, st>>>(xyzm, n, D, keys, idx);
    if ((rc = run_cub([&](void* t, size_t& b) {
             return cub::DeviceRadixSort::SortPairs(t, b, keys, keys_s, idx, idx_s, n, 0, int(3 * D), st);
         })))
        return rc;
    k_last_of_run<<<grid, 256, 0, st>>>(keys_s, n, flag);
    VE_BUILD_ALLOC(leaf_key, uint64_t, n);
    VE_BUILD_ALLOC(leaf_idx, uint32_t, n);
    if ((rc = run_cub([&](void* t, size_t& b) {
             return cub::DeviceSelect::Flagged(t, b, keys_s, flag, leaf_key, nsel, n, st);
         })) ||
        (rc = run_cub([&](void* t, size_t& b) {
             return cub::DeviceSelect::Flagged(t, b, idx_s, flag, leaf_idx, nsel, n, st);
         })))
        return rc;
    uint64_t nu = 0;
    VE_CUDA(cudaMemcpyAsync(&nu, nsel, 8, cudaMemcpyDeviceToHost, st));
    VE_CUDA(cudaStreamSynchronize(st));
    if (nu == 0) return empty_scene();
    VE_BUILD_ALLOC(leaf_mat, uint32_t, nu);
    k_gather_material<<<grid, 256, 0, st>>>(xyzm, leaf_idx, nu, leaf_mat);
    // 2. internal levels D .. 2 (level l: prefixes of l-1 digits)
    struct Level {
        uint64_t* prefix = nullptr;
        uint32_t* count = nullptr;
        uint32_t* parent_of = nullptr;  // 1-based index of each node's parent in level l-1 (l >= 3)
        uint64_t m = 0;
    };
    std::vector<Level> lv(D + 2);
    lv[D + 1].prefix = leaf_key;
    lv[D + 1].m = nu;
    for (uint32_t l = D + 1; l >= 3; l--) {
        const uint64_t m = lv[l].m;
        VE_BUILD_ALLOC(par, uint64_t, m);
        VE_BUILD_ALLOC(head, uint32_t, m);
        VE_BUILD_ALLOC(scan, uint32_t, m);
        VE_BUILD_ALLOC(uniq, uint64_t, m);
        VE_BUILD_ALLOC(cnt, uint32_t, m);
        k_prefix_heads<<<grid, 256, 0, st>>>(lv[l].prefix, m, 3u, par, head);
        if ((rc = run_cub([&](void* t, size_t& b) {
                 return cub::DeviceRunLengthEncode::Encode(t, b, par, uniq, cnt, nsel, m, st);
             })) ||
            (rc = run_cub([&](void* t, size_t& b) { return cub::DeviceScan::InclusiveSum(t, b, head, scan, m, st); })))
            return rc;
        lv[l].parent_of = scan;
        uint64_t mp = 0;
        VE_CUDA(cudaMemcpyAsync(&mp, nsel, 8, cudaMemcpyDeviceToHost, st));
        VE_CUDA(cudaStreamSynchronize(st));
        lv[l - 1].prefix = uniq;
        lv[l - 1].count = cnt;
        lv[l - 1].m = mp;
    }
    uint64_t M = 0;
    std::vector<uint64_t> base(D + 2, 0);
    for (uint32_t l = 2; l <= D; l++) {
        base[l] = M;
        M += lv[l].m;
    }
    if (9ull + 8ull * M >= (1ull << 28)) return fail(VE_ERR_CAPACITY, "scene_build: node array exceeds 2^28 words");
    // 3. blocks: rank of every internal node (levels 2..D) in the stack order
    VE_BUILD_ALLOC(block, uint32_t, M);
    if (M) {
        VE_BUILD_ALLOC(okey, uint64_t, M);
        VE_BUILD_ALLOC(okey_s, uint64_t, M);
        VE_BUILD_ALLOC(oval, uint32_t, M);
        VE_BUILD_ALLOC(oval_s, uint32_t, M);
        for (uint32_t l = 2; l <= D; l++)
            k_order_keys<<<grid, 256, 0, st>>>(lv[l].prefix, lv[l].m, l - 1u, uint32_t(base[l]), okey + base[l],
                                                oval + base[l]);
        if ((rc = run_cub([&](void* t, size_t& b) {
                 return cub::DeviceRadixSort::SortPairs(t, b, okey, okey_s, oval, oval_s, M, 0, 64, st);
             })))
            return rc;
        k_scatter_rank<<<grid, 256, 0, st>>>(oval_s, M, block);
    }
    // 4. words
    const uint64_t size = 9ull + 8ull * M;
    void* a = nullptr;
    if (cudaMalloc(&a, (size + 8) * 4) != cudaSuccess)
        return fail(VE_ERR_NOMEM, "scene_build: node array allocation failed");
    uint32_t* w = reinterpret_cast<uint32_t*>(a) + 7;
    cudaMemsetAsync(a, 0, (size + 8) * 4, st);
    k_root_word<<<1, 1, 0, st>>>(uint32_t(lv[2].m), w);
    for (uint32_t l = 2; l <= D + 1; l++) {
        const bool leaf = l == D + 1;
        const uint32_t* pb = l >= 3 ? block + base[l - 1] - 1 : nullptr;  // parent_of is 1-based
        k_level_words<<<grid, 256, 0, st>>>(lv[l].prefix, lv[l].m, lv[l].parent_of, pb,
                                             leaf ? nullptr : block + base[l], lv[l].count, leaf ? leaf_mat : nullptr, w);
    }
    const cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        cudaFree(a);
        return fail(VE_ERR_CUDA, std::string("scene_build: ") + cudaGetErrorString(e));
    }
    *alloc = a;
    *words = w;
    *n_words = size;
    return VE_OK;
}

}  // namespace ve

extern "C" {

int ve_scene_build(ve_ctx* c, const uint32_t* xyzm, uint64_t n, uint32_t depth, uint32_t flags, int32_t* scene_id,
                   uint64_t* n_words) {
    if (c) join_alt(c);  // after the second frame set's frames in flight
    if (!c || (!xyzm && n) || !scene_id) return fail(VE_ERR_INVALID, "scene_build: null argument");
    if (depth < 1 || depth > 16) return fail(VE_ERR_INVALID, "scene_build: depth must be in [1, 16]");
    if (n >= (1ull << 32)) return fail(VE_ERR_CAPACITY, "scene_build: at most 2^32 - 1 voxels");
    const uint64_t L = 1ull << depth;
    for (uint64_t i = 0; i < n; i++) {
        if (xyzm[4 * i] >= L || xyzm[4 * i + 1] >= L || xyzm[4 * i + 2] >= L)
            return fail(VE_ERR_INVALID, "scene_build: voxel outside the 2^depth cube");
        if (xyzm[4 * i + 3] == 0u || xyzm[4 * i + 3] > 127u)
            return fail(VE_ERR_INVALID, "scene_build: materials are 1..127");
    }
    cudaSetDevice(c->device);
    uint32_t* d_in = nullptr;
    if (cudaMalloc(&d_in, std::max<uint64_t>(n, 1) * 16) != cudaSuccess)
        return fail(VE_ERR_NOMEM, "scene_build: device allocation failed");
    if (n) VE_CUDA(cudaMemcpyAsync(d_in, xyzm, n * 16, cudaMemcpyHostToDevice, c->stream));
    SceneSlot s;
    s.depth = depth;
    int rc = build_scene_words(c, d_in, n, depth, &s.alloc, &s.nodes, &s.n_words);
    cudaStreamSynchronize(c->stream);
    cudaFree(d_in);
    if (rc) return rc;
    const size_t cache_bytes = sizeof(CacheEntry) << c->cfg.hash_log2;
    if (cudaMalloc(&s.cache, cache_bytes) != cudaSuccess) {
        cudaFree(s.alloc);
        return fail(VE_ERR_NOMEM, "scene_build: radiance cache allocation failed");
    }
    VE_CUDA(cudaMemsetAsync(s.cache, 0, cache_bytes, c->stream));
    s.live = true;
    if ((rc = build_top(c, s)) || (!(flags & VE_SCENE_KEEP_NORMALS) && (rc = compute_normals(c, s)))) {
        cudaFree(s.alloc);
        cudaFree(s.cache);
        if (s.top) cudaFree(s.top);
        return rc;
    }
    VE_CUDA(cudaStreamSynchronize(c->stream));
    int32_t id = -1;
    for (size_t i = 0; i < c->scenes.size(); i++)
        if (!c->scenes[i].live) {
            id = int32_t(i);
            break;
        }
    if (id < 0) {
        id = int32_t(c->scenes.size());
        c->scenes.push_back(s);
    } else {
        c->scenes[id] = s;
    }
    c->scenes_dirty = true;
    c->gen++;
    *scene_id = id;
    if (n_words) *n_words = s.n_words;
    return VE_OK;
}

int ve_scene_upload(ve_ctx* c, const uint32_t* words, uint64_t n_words, uint32_t depth, uint32_t flags,
                    int32_t* scene_id) {
    if (c) join_alt(c);  // after the second frame set's frames in flight
    if (!c || !words || !scene_id) return fail(VE_ERR_INVALID, "scene_upload: null argument");
    if (n_words < 9) return fail(VE_ERR_INVALID, "scene_upload: a node array has at least 9 words");
    if (depth < 1 || depth > 16) return fail(VE_ERR_INVALID, "scene_upload: depth must be in [1, 16]");
    if (n_words >= (1ull << 32)) return fail(VE_ERR_CAPACITY, "scene_upload: more than 2^32 words");
    cudaSetDevice(c->device);
    SceneSlot s;
    s.depth = depth;
    s.n_words = n_words;
    // nodes start 7 words into the allocation so every 8-child block
    // (slots 1 + 8k) begins on a 32-byte boundary
    if (cudaMalloc(&s.alloc, (n_words + 8) * 4) != cudaSuccess)
        return fail(VE_ERR_NOMEM, "scene_upload: node array allocation failed");
    s.nodes = reinterpret_cast<uint32_t*>(s.alloc) + 7;
    const size_t cache_bytes = sizeof(CacheEntry) << c->cfg.hash_log2;
    if (cudaMalloc(&s.cache, cache_bytes) != cudaSuccess) {
        cudaFree(s.alloc);
        return fail(VE_ERR_NOMEM, "scene_upload: radiance cache allocation failed");
    }
    VE_CUDA(cudaMemcpyAsync(s.nodes, words, n_words * 4, cudaMemcpyHostToDevice, c->stream));
    VE_CUDA(cudaMemsetAsync(s.cache, 0, cache_bytes, c->stream));
    s.live = true;
    if (int rc = build_top(c, s)) {
        cudaFree(s.alloc);
        cudaFree(s.cache);
        if (s.top) cudaFree(s.top);
        return rc;
    }
    if (!(flags & VE_SCENE_KEEP_NORMALS)) {
        int rc = compute_normals(c, s);
        if (rc) {
            cudaFree(s.alloc);
            cudaFree(s.cache);
            if (s.top) cudaFree(s.top);
            return rc;
        }
    }
    VE_CUDA(cudaStreamSynchronize(c->stream));
    int32_t id = -1;
    for (size_t i = 0; i < c->scenes.size(); i++)
        if (!c->scenes[i].live) { id = int32_t(i); break; }
    if (id < 0) {
        id = int32_t(c->scenes.size());
        c->scenes.push_back(s);
    } else {
        c->scenes[id] = s;
    }
    c->scenes_dirty = true;
    c->gen++;
    *scene_id = id;
    return VE_OK;
}

int ve_scene_release(ve_ctx* c, int32_t id) {
    if (c) join_alt(c);  // after the second frame set's frames in flight
    if (!c || id < 0 || size_t(id) >= c->scenes.size() || !c->scenes[id].live)
        return fail(VE_ERR_NOT_FOUND, "scene_release: unknown scene");
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    SceneSlot& s = c->scenes[id];
    cudaFree(s.alloc);
    cudaFree(s.cache);
    if (s.top) cudaFree(s.top);
    if (s.rank) cudaFree(s.rank);
    if (s.lbuf) cudaFree(s.lbuf);
    if (s.ntab) cudaFree(s.ntab);
    free_emissive(s);
    s = SceneSlot();
    c->scenes_dirty = true;
    c->gen++;
    return VE_OK;
}

int ve_scene_apply_edits(ve_ctx* c, int32_t id, const uint32_t* slots, const uint32_t* words, uint64_t n,
                         uint32_t flags) {
    if (c) join_alt(c);  // after the second frame set's frames in flight
    if (!c || id < 0 || size_t(id) >= c->scenes.size() || !c->scenes[id].live)
        return fail(VE_ERR_NOT_FOUND, "scene_apply_edits: unknown scene");
    if (n && (!slots || !words)) return fail(VE_ERR_INVALID, "scene_apply_edits: null arrays");
    SceneSlot& s = c->scenes[id];
    for (uint64_t i = 0; i < n; i++)
        if (slots[i] >= s.n_words) return fail(VE_ERR_CAPACITY, "scene_apply_edits: slot beyond the uploaded array");
    cudaSetDevice(c->device);
    if (n) {  // one copy of the (slot, word) lists, one scatter
        uint32_t* d = nullptr;
        if (cudaMalloc(&d, n * 8) != cudaSuccess) return fail(VE_ERR_NOMEM, "scene_apply_edits: allocation failed");
        cudaMemcpyAsync(d, slots, n * 4, cudaMemcpyHostToDevice, c->stream);
        cudaMemcpyAsync(d + n, words, n * 4, cudaMemcpyHostToDevice, c->stream);
        k_scatter_words<<<c->num_sms * 4, 256, 0, c->stream>>>(s.nodes, d, d + n, n);
        const cudaError_t e = cudaStreamSynchronize(c->stream);
        cudaFree(d);
        if (e != cudaSuccess) return fail(VE_ERR_CUDA, std::string("scene_apply_edits: ") + cudaGetErrorString(e));
    }
    if (int rc = build_top(c, s)) return rc;
    if (!(flags & VE_SCENE_KEEP_NORMALS)) {
        int rc = compute_normals(c, s);
        if (rc) return rc;
    }
    VE_CUDA(cudaStreamSynchronize(c->stream));
    return VE_OK;
}

int ve_scene_refresh(ve_ctx* c, int32_t id, const uint32_t* xyz, uint64_t n, uint32_t flags) {
    if (c) join_alt(c);  // after the second frame set's frames in flight
    if (!c || id < 0 || size_t(id) >= c->scenes.size() || !c->scenes[id].live)
        return fail(VE_ERR_NOT_FOUND, "scene_refresh: unknown scene");
    if (n && !xyz) return fail(VE_ERR_INVALID, "scene_refresh: null positions");
    if (n > (1ull << 26)) return fail(VE_ERR_CAPACITY, "scene_refresh: at most 2^26 positions per call");
    SceneSlot& s = c->scenes[id];
    if (s.normal_radius)
        return fail(VE_ERR_STATE, "scene_refresh: a ball-normal scene recomputes its normals with "
                                  "ve_scene_apply_edits (without VE_SCENE_KEEP_NORMALS) or ve_scene_normal_mode");
    const uint32_t L = 1u << s.depth;
    for (uint64_t i = 0; i < 3 * n; i++)
        if (xyz[i] >= L) return fail(VE_ERR_INVALID, "scene_refresh: position outside the scene");
    if (n == 0) return VE_OK;
    cudaSetDevice(c->device);
    uint32_t* d = nullptr;
    if (cudaMalloc(&d, n * 12) != cudaSuccess) return fail(VE_ERR_NOMEM, "scene_refresh: allocation failed");
    cudaMemcpyAsync(d, xyz, n * 12, cudaMemcpyHostToDevice, c->stream);
    k_refresh<<<c->num_sms * 8, 256, 0, c->stream>>>(s.nodes, s.n_words, s.depth, d, n,
                                                     (flags & VE_REFRESH_KEEP_CACHE) ? nullptr : s.cache,
                                                     c->cfg.hash_log2, c->cfg.hash_probes);
    const cudaError_t e = cudaStreamSynchronize(c->stream);
    cudaFree(d);
    if (e != cudaSuccess) return fail(VE_ERR_CUDA, std::string("scene_refresh: ") + cudaGetErrorString(e));
    return VE_OK;
}

int ve_scene_normal_mode(ve_ctx* c, int32_t id, uint32_t radius) {
    if (c) join_alt(c);  // after the second frame set's frames in flight
    if (!c || id < 0 || size_t(id) >= c->scenes.size() || !c->scenes[id].live)
        return fail(VE_ERR_NOT_FOUND, "scene_normal_mode: unknown scene");
    if (radius > VE_NORMAL_BALL_MAX_RADIUS)
        return fail(VE_ERR_INVALID, "scene_normal_mode: radius above VE_NORMAL_BALL_MAX_RADIUS");
    SceneSlot& s = c->scenes[id];
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    s.normal_radius = radius;
    if (int rc = compute_normals(c, s)) return rc;
    return sync_scenes(c);
}

int ve_scene_download(ve_ctx* c, int32_t id, uint32_t* out, uint64_t cap, uint64_t* n_words) {
    if (c) join_alt(c);  // after the second frame set's frames in flight
    if (!c || id < 0 || size_t(id) >= c->scenes.size() || !c->scenes[id].live)
        return fail(VE_ERR_NOT_FOUND, "scene_download: unknown scene");
    SceneSlot& s = c->scenes[id];
    if (n_words) *n_words = s.n_words;
    if (out && cap) {
        VE_CUDA(cudaMemcpyAsync(out, s.nodes, std::min<uint64_t>(cap, s.n_words) * 4, cudaMemcpyDeviceToHost, c->stream));
        VE_CUDA(cudaStreamSynchronize(c->stream));
    }
    return VE_OK;
}

// ve_raycast_batch: rays from host memory through k_raycast_batch.
int ve_raycast_batch(ve_ctx* c, int32_t id, const float* origins, const float* dirs, uint64_t n,
                     uint32_t controlchecks, uint32_t flags, uint32_t* out) {
    if (c) join_alt(c);  // after the second frame set's frames in flight
    if (!c || id < 0 || size_t(id) >= c->scenes.size() || !c->scenes[id].live)
        return fail(VE_ERR_NOT_FOUND, "raycast_batch: unknown scene");
    if (n == 0) return VE_OK;
    if (!origins || !dirs || !out) return fail(VE_ERR_INVALID, "raycast_batch: null argument");
    if (n > (1ull << 28)) return fail(VE_ERR_CAPACITY, "raycast_batch: at most 2^28 rays per call");
    if (controlchecks > kMaxControlChecks) return fail(VE_ERR_INVALID, "raycast_batch: controlchecks must be <= 65536");
    int rc;
    if ((rc = c->ray_in.ensure(6 * n)) || (rc = c->ray_out.ensure(8 * n))) return rc;
    const SceneSlot& sl = c->scenes[id];
    const DevScene S{sl.nodes, sl.n_words, sl.cache, sl.depth, c->cfg.hash_log2, c->cfg.hash_probes, sl.top_level, sl.top};
    cudaStream_t st = c->stream;
    VE_CUDA(cudaMemcpyAsync(c->ray_in.p, origins, 12 * n, cudaMemcpyHostToDevice, st));
    VE_CUDA(cudaMemcpyAsync(c->ray_in.p + 3 * n, dirs, 12 * n, cudaMemcpyHostToDevice, st));
    const uint32_t grid = uint32_t(std::min<uint64_t>((n + 255) / 256, uint64_t(c->num_sms) * 16));
    if (flags & VE_RAYCAST_FULL_WALK)
        k_raycast_batch<true><<<grid, 256, 0, st>>>(S, c->ray_in.p, n, controlchecks, c->ray_out.p);
    else
        k_raycast_batch<false><<<grid, 256, 0, st>>>(S, c->ray_in.p, n, controlchecks, c->ray_out.p);
    VE_CUDA(cudaGetLastError());
    VE_CUDA(cudaMemcpyAsync(out, c->ray_out.p, 32 * n, cudaMemcpyDeviceToHost, st));
    VE_CUDA(cudaStreamSynchronize(st));
    return VE_OK;
}

int ve_scene_footprint(ve_ctx* c, int32_t id, uint64_t* bytes) {
    if (!c || !bytes || id < 0 || size_t(id) >= c->scenes.size() || !c->scenes[id].live)
        return fail(VE_ERR_NOT_FOUND, "scene_footprint: unknown scene");
    const SceneSlot& sl = c->scenes[id];
    const uint64_t top = sl.top_level ? (4ull << (3u * (sl.top_level - 1u))) : 0ull;
    *bytes = (sl.n_words + 8) * 4 + (sizeof(CacheEntry) << c->cfg.hash_log2) + top;
    return VE_OK;
}

int ve_scene_clip_box(ve_ctx* c, int32_t id, float lo[3], float hi[3], uint32_t* bounded) {
    if (!c || id < 0 || size_t(id) >= c->scenes.size() || !c->scenes[id].live)
        return fail(VE_ERR_NOT_FOUND, "scene_clip_box: unknown scene");
    if (!lo || !hi || !bounded) return fail(VE_ERR_INVALID, "scene_clip_box: null argument");
    const SceneSlot& sl = c->scenes[id];
    for (int a = 0; a < 3; a++) {
        lo[a] = sl.clip_lo[a];
        hi[a] = sl.clip_hi[a];
    }
    *bounded = sl.clip_lo[0] > -1e29f ? 1u : 0u;
    return VE_OK;
}

int ve_set_materials(ve_ctx* c, const void* entries, uint32_t n) {
    if (c) join_alt(c);  // after the second frame set's frames in flight
    if (!c || (!entries && n)) return fail(VE_ERR_INVALID, "set_materials: null argument");
    if (n > 128) return fail(VE_ERR_CAPACITY, "set_materials: at most 128 materials");
    std::vector<DevMaterial> m(128);
    std::memset(m.data(), 0, m.size() * sizeof(DevMaterial));
    const uint8_t* src = static_cast<const uint8_t*>(entries);
    for (uint32_t i = 0; i < n; i++) {
        float f[16];
        std::memcpy(f, src + 64 * i, 64);
        int32_t emissive;
        std::memcpy(&emissive, src + 64 * i + 44, 4);
        m[i].albedo_rough = make_float4(f[0], f[1], f[2], f[8]);
        m[i].params = make_float4(f[10], f[9], emissive ? 1.0f : 0.0f, f[12]);
    }
    cudaSetDevice(c->device);
    VE_CUDA(cudaMemcpyAsync(c->d_mats.p, m.data(), 128 * sizeof(DevMaterial), cudaMemcpyHostToDevice, c->stream));
    VE_CUDA(cudaStreamSynchronize(c->stream));
    return VE_OK;
}

int ve_cache_reset(ve_ctx* c, int32_t id) {
    if (c) join_alt(c);  // after the second frame set's frames in flight
    if (!c || id < 0 || size_t(id) >= c->scenes.size() || !c->scenes[id].live)
        return fail(VE_ERR_NOT_FOUND, "cache_reset: unknown scene");
    VE_CUDA(cudaMemsetAsync(c->scenes[id].cache, 0, sizeof(CacheEntry) << c->cfg.hash_log2, c->stream));
    // the emissive lights and reservoirs go with it, and the lBuffer
    if (int rc = reset_emissive(c, c->scenes[id])) return rc;
    if (c->scenes[id].lbuf) {
        VE_CUDA(cudaMemsetAsync(c->scenes[id].lbuf, 0, kLbBytes, c->stream));
        VE_CUDA(cudaStreamSynchronize(c->stream));
    }
    // the scheduling thresholds derive from the cache: forget them too
    if (c->scenes[id].rank) {
        const int rc = reset_rank(c, c->scenes[id].rank);
        if (rc) return rc;
    }
    VE_CUDA(cudaStreamSynchronize(c->stream));
    return VE_OK;
}

int ve_lbuffer_dump(ve_ctx* c, int32_t id, uint32_t* out, uint64_t cap, uint64_t* n) {
    if (c) join_alt(c);  // after the second frame set's frames in flight
    if (!c || id < 0 || size_t(id) >= c->scenes.size() || !c->scenes[id].live)
        return fail(VE_ERR_NOT_FOUND, "lbuffer_dump: unknown scene");
    const SceneSlot& s = c->scenes[id];
    if (n) *n = 0;
    if (!s.lbuf) return VE_OK;
    std::vector<uint32_t> h(kLbBytes / sizeof(uint32_t));
    VE_CUDA(cudaMemcpyAsync(h.data(), s.lbuf, kLbBytes, cudaMemcpyDeviceToHost, c->stream));
    VE_CUDA(cudaStreamSynchronize(c->stream));
    uint64_t k = 0;
    for (uint32_t r = 0; r < kLbWidth; r++)
        for (uint32_t i = 0; i < kLbSlots; i++) {
            const uint32_t* w = h.data() + (size_t(r) * kLbSlots + i) * kLbStride;
            if (w[0] == 0u) continue;
            if (out && k < cap) {
                uint32_t* o = out + 14 * k;
                o[0] = r;
                o[1] = i;
                std::memcpy(o + 2, w, kLbStride * sizeof(uint32_t));
            }
            k++;
        }
    if (n) *n = k;
    return VE_OK;
}

int ve_cache_dump(ve_ctx* c, int32_t id, uint32_t* vids, uint32_t* counts, float* values, uint64_t cap, uint64_t* n) {
    if (c) join_alt(c);  // after the second frame set's frames in flight
    if (!c || id < 0 || size_t(id) >= c->scenes.size() || !c->scenes[id].live)
        return fail(VE_ERR_NOT_FOUND, "cache_dump: unknown scene");
    const size_t N = size_t(1) << c->cfg.hash_log2;
    std::vector<CacheEntry> h(N);
    VE_CUDA(cudaMemcpyAsync(h.data(), c->scenes[id].cache, N * sizeof(CacheEntry), cudaMemcpyDeviceToHost, c->stream));
    VE_CUDA(cudaStreamSynchronize(c->stream));
    std::vector<size_t> idx;
    for (size_t i = 0; i < N; i++)
        if (h[i].key) idx.push_back(i);
    std::sort(idx.begin(), idx.end(), [&](size_t a, size_t b) { return h[a].key < h[b].key; });
    if (n) *n = idx.size();
    for (size_t j = 0; j < idx.size() && j < cap; j++) {
        const CacheEntry& e = h[idx[j]];
        if (vids) vids[j] = e.key;
        if (counts) counts[j] = e.count;
        if (values) {
            values[5 * j] = e.rgbw.w;
            values[5 * j + 1] = e.rgbw.x;
            values[5 * j + 2] = e.rgbw.y;
            values[5 * j + 3] = e.rgbw.z;
            values[5 * j + 4] = e.l2;
        }
    }
    return VE_OK;
}

int ve_render(ve_ctx* c, const ve_view* view, ve_frame_outputs* out) {
    if (!c || !view) return fail(VE_ERR_INVALID, "render: null argument");
    cudaSetDevice(c->device);
    return render_batch(c, view, 1, out);
}

int ve_render_batch(ve_ctx* c, const ve_view* views, uint32_t n, ve_frame_outputs* outs) {
    if (!c) return fail(VE_ERR_INVALID, "render_batch: null context");
    cudaSetDevice(c->device);
    return render_batch(c, views, n, outs);
}

// A device range [p, p + bytes) inside one allocation of this context's
// device (split-frame record buffers come from the caller).
static int check_device_range(ve_ctx* c, const void* p, uint64_t bytes, const char* what) {
    if (bytes == 0) return VE_OK;
    if (!p) return fail(VE_ERR_INVALID, std::string(what) + ": null device pointer");
    if (uintptr_t(p) % 16u) return fail(VE_ERR_INVALID, std::string(what) + ": records must be 16-byte aligned");
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess || at.devicePointer == nullptr ||
        (at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged) || at.device != c->device) {
        cudaGetLastError();
        return fail(VE_ERR_INVALID, std::string(what) + ": not device memory of the context's GPU");
    }
    using RangeFn = CUresult (*)(CUdeviceptr*, size_t*, CUdeviceptr);
    static const RangeFn range = []() -> RangeFn {  // looked up once (thread-safe static init)
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPointByVersion("cuMemGetAddressRange", &fn, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            return reinterpret_cast<RangeFn>(fn);
        return nullptr;
    }();
    if (!range) return fail(VE_ERR_CUDA, std::string(what) + ": cannot query allocation ranges");
    CUdeviceptr base = 0;
    size_t size = 0;
    if (range(&base, &size, CUdeviceptr(uintptr_t(p))) != CUDA_SUCCESS)
        return fail(VE_ERR_INVALID, std::string(what) + ": not a device allocation");
    if (uintptr_t(p) + bytes > uintptr_t(base) + size)
        return fail(VE_ERR_INVALID, std::string(what) + ": the records run past the end of their allocation");
    return VE_OK;
}

static int split_scene_ok(ve_ctx* c, int32_t id, const char* what) {
    if (!c || id < 0 || size_t(id) >= c->scenes.size() || !c->scenes[id].live)
        return fail(VE_ERR_NOT_FOUND, std::string(what) + ": unknown scene");
    if (c->split_scene != id || !c->split_delta.p)
        return fail(VE_ERR_STATE, std::string(what) + ": no VE_FRAME_SPLIT frame of this scene");
    return VE_OK;
}

int ve_split_export(ve_ctx* c, int32_t id, void* dev_out, uint64_t cap, uint64_t* n) {
    if (c) join_alt(c);  // after the second frame set's frames in flight
    if (int rc = split_scene_ok(c, id, "split_export")) return rc;
    if (!n) return fail(VE_ERR_INVALID, "split_export: null count");
    cudaSetDevice(c->device);
    const uint64_t N = uint64_t(1) << c->cfg.hash_log2;
    cap = std::min(cap, N);
    if (int rc = check_device_range(c, dev_out, cap * sizeof(ve_split_record), "split_export")) return rc;
    uint32_t* cnt = c->split_cnt.p;
    VE_CUDA(cudaMemsetAsync(cnt, 0, sizeof(uint32_t), c->stream));
    k_split_export<<<c->num_sms * 8, 256, 0, c->stream>>>(c->split_delta.p, uint32_t(N),
                                                          static_cast<uint4*>(dev_out), uint32_t(cap), cnt);
    VE_CUDA(cudaGetLastError());
    c->split_delta_clean = true;
    uint32_t h = 0;
    VE_CUDA(cudaMemcpyAsync(&h, cnt, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    VE_CUDA(cudaStreamSynchronize(c->stream));
    *n = h;
    return VE_OK;
}

int ve_split_merge(ve_ctx* c, int32_t id, const void* dev_parts, const uint64_t* counts, uint32_t n_parts,
                   uint64_t stride, uint64_t* dropped) {
    if (c) join_alt(c);  // after the second frame set's frames in flight
    if (int rc = split_scene_ok(c, id, "split_merge")) return rc;
    if (n_parts && !counts) return fail(VE_ERR_INVALID, "split_merge: null counts");
    // bounds that keep part offsets (k * stride records) far from overflow
    if (n_parts > 65536u) return fail(VE_ERR_INVALID, "split_merge: at most 65536 parts");
    if (stride > (uint64_t(1) << 36)) return fail(VE_ERR_INVALID, "split_merge: stride beyond any allocation");
    const uint64_t N = uint64_t(1) << c->cfg.hash_log2;
    uint64_t end = 0;
    for (uint32_t k = 0; k < n_parts; k++) {
        if (counts[k] > stride) return fail(VE_ERR_INVALID, "split_merge: a part holds more records than its stride");
        if (counts[k] > N) return fail(VE_ERR_INVALID, "split_merge: a part holds more records than a cache");
        if (counts[k]) end = std::max(end, uint64_t(k) * stride + counts[k]);
    }
    cudaSetDevice(c->device);
    if (int rc = check_device_range(c, dev_parts, end * sizeof(ve_split_record), "split_merge")) return rc;
    uint32_t* drop = c->split_cnt.p + 1;
    VE_CUDA(cudaMemsetAsync(drop, 0, sizeof(uint32_t), c->stream));
    const ve_split_record* base = static_cast<const ve_split_record*>(dev_parts);
    CacheEntry* cache = c->scenes[id].cache;
    for (uint32_t k = 0; k < n_parts; k++) {
        if (!counts[k]) continue;
        const uint32_t blocks = uint32_t(std::min<uint64_t>((counts[k] + 255) / 256, uint64_t(c->num_sms) * 8));
        k_split_merge<<<blocks, 256, 0, c->stream>>>(cache, c->cfg.hash_log2, c->cfg.hash_probes,
                                                     reinterpret_cast<const uint4*>(base + uint64_t(k) * stride),
                                                     uint32_t(counts[k]), drop);
    }
    VE_CUDA(cudaGetLastError());
    uint32_t h = 0;
    VE_CUDA(cudaMemcpyAsync(&h, drop, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    VE_CUDA(cudaStreamSynchronize(c->stream));
    if (dropped) *dropped = h;
    return VE_OK;
}

int ve_split_resolve(ve_ctx* c, const ve_view* view, ve_frame_outputs* out) {
    if (c) join_alt(c);  // after the second frame set's frames in flight
    if (!c || !view) return fail(VE_ERR_INVALID, "split_resolve: null argument");
    if (int rc = split_scene_ok(c, view->scene_id, "split_resolve")) return rc;
    const ve_frame_config& f = view->frame;
    const ve_frame_config& g = c->split_frame;
    if (!(f.flags & VE_FRAME_SPLIT) || f.width != g.width || f.height != g.height || f.row_begin != g.row_begin ||
        f.row_end != g.row_end || f.reconstruction_radius != g.reconstruction_radius)
        return fail(VE_ERR_STATE, "split_resolve: the view is not the one of the last VE_FRAME_SPLIT frame");
    if (f.render_type > VE_RENDER_VARIANCE) return fail(VE_ERR_INVALID, "split_resolve: unknown render type");
    cudaSetDevice(c->device);
    const uint32_t tiles = ((f.width + 15) / 16) * ((f.height + 15) / 16);
    const int slot = c->staging_next;
    c->staging_next = (slot + 1) % ve_ctx::kStaging;
    VE_CUDA(cudaEventSynchronize(c->staging_ev[slot]));
    DevView* hv = c->h_views[slot];
    fill_view(hv[0], *view);
    cudaStream_t st = c->stream;
    if (c->copy_stream) VE_CUDA(cudaStreamWaitEvent(st, c->copy_done[0], 0));  // an async copy of set 0
    VE_CUDA(cudaMemcpyAsync(c->d_views.p, hv, sizeof(DevView), cudaMemcpyHostToDevice, st));
    VE_CUDA(cudaEventRecord(c->staging_ev[slot], st));
    FrameArgs a{};
    a.views = c->d_views.p;
    a.n_views = 1;
    a.total_tiles = tiles;
    a.scenes = c->d_scenes.p;
    a.mats = c->d_mats.p;
    a.gbuf = c->gbuf.p;
    a.out_vid = c->out_vid.p; a.out_node = c->out_node.p;
    a.out_rgb = c->out_rgb.p; a.out_mapped = c->out_mapped.p; a.out_mapped8 = c->out_m8.p;
    k_resolve<<<tiles, 256, 0, st>>>(a);
    VE_CUDA(cudaGetLastError());
    uint64_t d2h = 0;
    if (out) {
        const uint64_t r0 = uint64_t(f.row_begin) * f.width, nr = uint64_t(f.row_end - f.row_begin) * f.width;
        if (out->gbuffer) { VE_CUDA(cudaMemcpyAsync(out->gbuffer + 4 * r0, c->gbuf.p + r0, nr * 16, cudaMemcpyDeviceToHost, st)); d2h += nr * 16; }
        if (out->voxel_id) { VE_CUDA(cudaMemcpyAsync(out->voxel_id + r0, c->out_vid.p + r0, nr * 4, cudaMemcpyDeviceToHost, st)); d2h += nr * 4; }
        if (out->hit_node) { VE_CUDA(cudaMemcpyAsync(out->hit_node + r0, c->out_node.p + r0, nr * 4, cudaMemcpyDeviceToHost, st)); d2h += nr * 4; }
        if (out->rgb) { VE_CUDA(cudaMemcpyAsync(out->rgb + 3 * r0, c->out_rgb.p + 3 * r0, nr * 12, cudaMemcpyDeviceToHost, st)); d2h += nr * 12; }
        if (out->mapped) { VE_CUDA(cudaMemcpyAsync(out->mapped + 3 * r0, c->out_mapped.p + 3 * r0, nr * 12, cudaMemcpyDeviceToHost, st)); d2h += nr * 12; }
        if (out->mapped8) { VE_CUDA(cudaMemcpyAsync(out->mapped8 + r0, c->out_m8.p + r0, nr * 4, cudaMemcpyDeviceToHost, st)); d2h += nr * 4; }
    }
    VE_CUDA(cudaStreamSynchronize(st));
    c->tot_h2d += sizeof(DevView);
    c->tot_d2h += d2h;
    return VE_OK;
}

int ve_get_launch_config(ve_ctx* c, ve_launch_config* cfg) {
    if (!c || !cfg) return fail(VE_ERR_INVALID, "get_launch_config: null argument");
    *cfg = c->launch;
    return VE_OK;
}

int ve_set_launch_config(ve_ctx* c, const ve_launch_config* cfg) {
    if (!c || !cfg) return fail(VE_ERR_INVALID, "set_launch_config: null argument");
    if (cfg->refill_threshold > 32) return fail(VE_ERR_INVALID, "set_launch_config: refill_threshold must be <= 32");
    c->launch = *cfg;
    apply_launch(c);
    return VE_OK;
}

int ve_autotune(ve_ctx* c, const ve_view* views, uint32_t nv, uint32_t frames, ve_launch_config* best) {
    if (c) join_alt(c);  // after the second frame set's frames in flight
    if (!c || !views || nv == 0) return fail(VE_ERR_INVALID, "autotune: no views");
    if (frames == 0) frames = 2;
    cudaSetDevice(c->device);
    std::vector<ve_view> tv(views, views + nv);
    for (auto& v : tv) v.frame.flags = (v.frame.flags | VE_FRAME_TIMING) & ~VE_FRAME_PATH_RGB;
    auto measure = [&](const ve_launch_config& cfg, float* ms) -> int {
        c->launch = cfg;
        apply_launch(c);
        int rc = render_batch(c, tv.data(), nv, nullptr);  // warm-up at this shape
        if (rc) return rc;
        VE_CUDA(cudaStreamSynchronize(c->stream));
        collect_all_timing(c);
        const float t0 = c->tot_ms[0];
        for (uint32_t f = 0; f < frames; f++)
            if ((rc = render_batch(c, tv.data(), nv, nullptr))) return rc;
        VE_CUDA(cudaStreamSynchronize(c->stream));
        collect_all_timing(c);
        *ms = (c->tot_ms[0] - t0) / float(frames);
        return VE_OK;
    };
    ve_launch_config cur{uint32_t(c->occ_trace), uint32_t(c->occ_shade), ve::kDefaultRefill, 0};
    float best_ms = 0.0f;
    int rc = measure(cur, &best_ms);
    if (rc) return rc;
    // coordinate descent: trace blocks/SM, shade blocks/SM, refill threshold
    for (int tb = 1; tb <= c->occ_trace; tb++) {
        ve_launch_config t = cur;
        t.trace_blocks_per_sm = uint32_t(tb);
        float ms = 0;
        if ((rc = measure(t, &ms))) return rc;
        if (ms < best_ms) { best_ms = ms; cur = t; }
    }
    for (int sb = 1; sb <= c->occ_shade; sb++) {
        ve_launch_config t = cur;
        t.shade_blocks_per_sm = uint32_t(sb);
        float ms = 0;
        if ((rc = measure(t, &ms))) return rc;
        if (ms < best_ms) { best_ms = ms; cur = t; }
    }
    for (uint32_t thr : {4u, 8u, 12u, 16u, 20u, 24u, 28u}) {
        ve_launch_config t = cur;
        t.refill_threshold = thr;
        float ms = 0;
        if ((rc = measure(t, &ms))) return rc;
        if (ms < best_ms) { best_ms = ms; cur = t; }
    }
    c->launch = cur;
    apply_launch(c);
    if (best) *best = cur;
    return VE_OK;
}

static void fill_counters(ve_frame_stats& r, const unsigned long long* h) {
    r.rays_primary = h[ST_RAYS_PRIMARY];
    r.rays_bounce = h[ST_RAYS_BOUNCE];
    r.rays_shadow = h[ST_RAYS_SHADOW];
    r.fetch_nodes = h[ST_FETCH];
    r.paths = h[ST_PATHS];
    r.deposits = h[ST_DEPOSITS];
    r.deposits_dropped = h[ST_DROPPED];
    r.dda_steps = h[ST_STEPS];
    r.fetch_nodes_trace = h[ST_FETCH_TRACE];
    r.dda_steps_trace = h[ST_STEPS_TRACE];
    r.nrc_queries = h[ST_NRC_QUERIES];
    r.nrc_hash_terminated = h[ST_NRC_HASH];
    r.nrc_samples = h[ST_NRC_SAMPLES];
    r.scheduled_voxels = h[ST_SCHED_VOXELS];
    r.scheduled_paths = h[ST_SCHED_PATHS];
    r.emissive_lights = h[ST_EM_LIGHTS];
    r.nee_emissive = h[ST_EM_NEE];
    r.restir_commits = h[ST_RES_WRITES];
    r.shadow_shared = h[ST_SHADOW_SHARED];
}

int ve_get_total_stats(ve_ctx* c, ve_frame_stats* s) {
    if (!c || !s) return fail(VE_ERR_INVALID, "get_total_stats: null argument");
    unsigned long long h[ST_TOTAL];
    if (c->alt.stream) VE_CUDA(cudaStreamSynchronize(c->alt.stream));  // the second set's totals
    VE_CUDA(cudaMemcpyAsync(h, c->totals.p, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    VE_CUDA(cudaStreamSynchronize(c->stream));
    collect_all_timing(c);
    ve_frame_stats r{};
    fill_counters(r, h);
    r.frames = c->tot_frames;
    r.h2d_bytes = c->tot_h2d;
    r.d2h_bytes = c->tot_d2h;
    r.ms_total = c->tot_ms[0]; r.ms_primary = c->tot_ms[1]; r.ms_trace = c->tot_ms[2];
    r.ms_shade = c->tot_ms[3]; r.ms_resolve = c->tot_ms[4]; r.ms_decay = c->tot_ms[5];
    r.ms_learned = c->tot_ms_learned;
    r.kernel_launches = c->tot_launches;
    r.trace_launches = c->tot_trace_launches;
    r.cache_capacity = 1ull << c->cfg.hash_log2;
    *s = r;
    return VE_OK;
}

int ve_reset_total_stats(ve_ctx* c) {
    if (c) join_alt(c);  // after the second frame set's frames in flight
    if (!c) return fail(VE_ERR_INVALID, "reset_total_stats: null context");
    VE_CUDA(cudaMemsetAsync(c->totals.p, 0, ST_TOTAL * sizeof(unsigned long long), c->stream));
    VE_CUDA(cudaStreamSynchronize(c->stream));
    collect_all_timing(c);
    c->tot_frames = c->tot_h2d = c->tot_d2h = 0;
    c->tot_launches = c->tot_trace_launches = 0;
    for (float& m : c->tot_ms) m = 0.0f;
    c->tot_ms_learned = 0.0f;
    return VE_OK;
}

int ve_get_stats(ve_ctx* c, ve_frame_stats* s) {
    if (!c || !s) return fail(VE_ERR_INVALID, "get_stats: null argument");
    VE_CUDA(cudaStreamSynchronize(c->stream));
    if (c->alt.stream) VE_CUDA(cudaStreamSynchronize(c->alt.stream));
    collect_all_timing(c);
    ve_frame_stats r = c->last;
    const unsigned long long* h = c->last_set == 1 ? c->alt.h_stats : c->h_stats;  // the last frame's set
    fill_counters(r, h);
    r.frames = 1;
    r.h2d_bytes = c->last_h2d;
    r.d2h_bytes = c->last_d2h;
    r.kernel_launches = c->last_launches;
    r.trace_launches = c->last_trace_launches;
    r.cache_capacity = 1ull << c->cfg.hash_log2;
    *s = r;
    return VE_OK;
}

// Allocation-free variant of the leaf normal pass (see include/ve.h).  The
// scratch is the file-scope g_noalloc_scratch; its device address belongs to
// the context that loaded the module, so it is cached per device together
// with that context and looked up again (cudaGetSymbolAddress, with the
// device current) on the first call on a device and whenever the current
// context differs from the cached one (after cudaDeviceReset, or under
// another context the caller made current).
struct NoAllocSlot {
    void* ctx;
    void* ptr;
};
static NoAllocSlot g_noalloc_slot[64] = {};
static std::mutex g_noalloc_mu;
using CtxGetCurrentFn = CUresult (*)(CUcontext*);

// the calling thread's current driver context (null when none is current)
static void* noalloc_current_ctx() {
    static CtxGetCurrentFn fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<CtxGetCurrentFn>(f);
    }();
    CUcontext c = nullptr;
    if (!fn || fn(&c) != CUDA_SUCCESS) return nullptr;
    return c;
}

int ve_fill_normals_noalloc(uint32_t* words, uint64_t n_words, uint32_t depth, void* stream) {
    if (!words) return fail(VE_ERR_INVALID, "fill_normals_noalloc: null node array");
    if (n_words < 9 || n_words >= (1ull << 32))
        return fail(VE_ERR_INVALID, "fill_normals_noalloc: n_words must be in [9, 2^32)");
    if (depth < 1 || depth > kNoAllocMaxDepth)
        return fail(VE_ERR_CAPACITY, "fill_normals_noalloc: depth must be in [1, 7] (fixed device scratch of " +
                                         std::to_string(kNoAllocBytes) + " bytes)");
    int dev = 0;
    VE_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(VE_ERR_INVALID, "fill_normals_noalloc: device index out of range");
    void* base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        NoAllocSlot& slot = g_noalloc_slot[dev];
        void* ctx = noalloc_current_ctx();
        if (!slot.ptr || !ctx || ctx != slot.ctx) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess)
                return fail(VE_ERR_CUDA, std::string("fill_normals_noalloc: cudaGetSymbolAddress: ") +
                                             cudaGetErrorString(e));
            // the lookup makes the device's primary context current when none was
            slot.ctx = ctx ? ctx : noalloc_current_ctx();
            slot.ptr = p;
        }
        base = slot.ptr;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned char* b = static_cast<unsigned char*>(base);
    uint32_t* cnt = reinterpret_cast<uint32_t*>(b);
    unsigned long long* fa = reinterpret_cast<unsigned long long*>(b + kNoAllocCounterBytes);
    unsigned long long* fb = fa + kNoAllocFrontier;
    uint32_t* occ = reinterpret_cast<uint32_t*>(fb + kNoAllocFrontier);
    // the array keeps the previous call's contents: clear counters and bitmask
    VE_CUDA(cudaMemsetAsync(cnt, 0, kNoAllocCounterBytes, st));
    VE_CUDA(cudaMemsetAsync(occ, 0, ((1ull << (3 * depth)) + 31) / 32 * 4, st));
    k_noalloc_seed<<<1, 32, 0, st>>>(cnt, fa);
    int n_sms = 148;
    cudaDeviceGetAttribute(&n_sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = n_sms * 8;
    unsigned long long* in = fa;
    unsigned long long* out = fb;
    for (uint32_t k = 0; k + 1 < depth; k++) {
        k_expand<<<grid, 256, 0, st>>>(words, n_words, depth, k, in, cnt + k, out, cnt + k + 1,
                                        uint32_t(kNoAllocFrontier));
        std::swap(in, out);
    }
    const uint32_t* lc = cnt + (depth - 1);
    k_leaf_pass<<<grid, 256, 0, st>>>(words, n_words, depth, in, lc, occ, 0, uint32_t(kNoAllocFrontier));
    k_leaf_pass<<<grid, 256, 0, st>>>(words, n_words, depth, in, lc, occ, 1, uint32_t(kNoAllocFrontier));
    VE_CUDA(cudaGetLastError());
    return VE_OK;
}

}  // extern "C"

#include "serve.cuh"
