/* ve.h — C ABI of the B200-native voxel ray pipeline (drop-in for the
 * RayPass / bounce-shade / AccumPass / AvgPass passes of
 * AnghelusAndrei/VoxelEngine3.0).
 *
 * Plain pointers and sizes only.  Every function returns an int status
 * (VE_OK = 0, negative = error); ve_last_error() gives the message of the
 * calling thread's last failure.  The caller owns every host array; the
 * library owns all device memory.  A context serialises its work on one CUDA
 * stream and is used from one host thread at a time.
 *
 * Each declaration names the reference interface it replaces
 * (paths relative to the reference repository).
 */
#ifndef VE_H
#define VE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define VE_OK 0
#define VE_ERR_INVALID (-1)  /* bad argument */
#define VE_ERR_CUDA (-2)     /* CUDA runtime error (message in ve_last_error) */
#define VE_ERR_NOMEM (-3)    /* allocation failed */
#define VE_ERR_CAPACITY (-4) /* a fixed capacity would be exceeded */
#define VE_ERR_NOT_FOUND (-5)
#define VE_ERR_TIMEOUT (-6) /* a bounded device wait gave up */
#define VE_ERR_STATE (-7)   /* call not valid in the current state */

/* ---- render types (src/renderer/core.hpp:71-78) ----------------------- */
#define VE_RENDER_DEFAULT 0
#define VE_RENDER_STRUCTURE 1
#define VE_RENDER_ALBEDO 2
#define VE_RENDER_NORMAL 3
#define VE_RENDER_VOXELID 4
#define VE_RENDER_VARIANCE 5

/* ---- flags ------------------------------------------------------------ */
#define VE_SCENE_KEEP_NORMALS 1u  /* upload words as given (no device normal pass) */
#define VE_FRAME_TIMING 1u        /* per-pass CUDA-event times into ve_frame_stats */
#define VE_FRAME_COUNT_FETCH 2u   /* count node-word fetches on the device */
#define VE_FRAME_PATH_RGB 4u      /* keep every path's deposit value (debug) */
#define VE_FRAME_LEARNED 8u       /* end paths at their second vertex with the scene's learned cache */
#define VE_FRAME_TERMINATE_HASH 16u /* end paths at their second vertex with the hashed per-voxel cache */
#define VE_FRAME_TRAIN 32u        /* record training samples and train the scene's learned cache */
#define VE_FRAME_EMISSIVE 128u    /* NEE toward the scene's emissive voxels instead of the sun: light
                                     registry, single-pick RIS and ReSTIR DI (shade.comp:576-836) */
#define VE_FRAME_LBUFFER 256u    /* the reference's dual-channel lBuffer AccumPass (shade.comp:96-257)
                                     in place of the FP32 per-voxel cache; one view per call */
#define VE_FRAME_SCHEDULED 64u    /* importance-aware voxel scheduling (schedule/rank/threshold.comp)
                                     in place of spp paths per pixel; single-view calls */
#define VE_FRAME_SPLIT 512u       /* one band of rows of a frame split across ranks: paths start only
                                     on rows [row_begin, row_end) and deposit into a per-frame table
                                     that ve_split_export / ve_split_merge exchange; the AvgPass runs
                                     in ve_split_resolve after the merge */
#define VE_FRAME_ASYNC_OUTPUTS 1024u /* host outputs (voxel_id, hit_node, rgb, mapped, mapped8 only) are copied on the
                                     context's copy stream while later frames render: the call returns
                                     once the frame is enqueued, and the host buffers (pinned memory for
                                     the copies to run asynchronously) hold the frame after
                                     ve_ctx_synchronize */
#define VE_CFG_NO_GRAPHS 1u       /* renderer config: enqueue kernels directly instead of
                                     replaying a CUDA graph of the frame's kernel sequence */
#define VE_CFG_PIPELINE 2u        /* renderer config: consecutive frames alternate between two sets of
                                     frame buffers on two streams, so that a frame's primary pass and
                                     first trace pass run while the previous frame finishes (its
                                     radiance-cache work still follows the previous frame's).  Applies
                                     to plain frames whose views all have bounces >= 1 and none of the
                                     flags TIMING, COUNT_FETCH, PATH_RGB, SCHEDULED, EMISSIVE, LBUFFER,
                                     LEARNED, TRAIN, TERMINATE_HASH, SPLIT; other frames and every other
                                     call on the context run after the frames in flight.  Costs a
                                     second copy of the path state.  Work the caller enqueues on the
                                     context's stream is ordered after pipelined frames only after
                                     ve_ctx_join (or any other call on the context). */

/* RendererConfig (src/renderer/core.hpp:30-42) plus device sizing.  The
 * radiance cache replaces the lBuffer hash image (renderer.cpp:27-40):
 * 2^hash_log2 entries per scene, linear probing up to hash_probes. */
typedef struct ve_renderer_config {
    int32_t device;
    uint32_t hash_log2;   /* 22 -> 4,194,304 entries (32 B each) */
    uint32_t hash_probes; /* 64 */
    uint32_t flags;
} ve_renderer_config;

/* FrameConfig (src/renderer/core.hpp:83-158): the knobs the plain method
 * reads, plus the benchmark lighting (directional sun + constant sky). */
typedef struct ve_frame_config {
    uint32_t width, height;
    uint32_t spp;                   /* paths per hit pixel */
    uint32_t bounces;               /* secondary bounces; MAX_BOUNCES = bounces + 1 */
    uint32_t primary_controlchecks; /* core.hpp:85 */
    uint32_t bounce_controlchecks;  /* core.hpp:86 */
    uint32_t reconstruction_radius; /* core.hpp:87 */
    uint32_t render_type;           /* VE_RENDER_* */
    uint32_t frame_index;           /* emit.comp frameIdx */
    float sun_dir[3];               /* unit vector toward the sun */
    float sun_intensity;
    float sky[3];                   /* constant sky radiance */
    float decay;                    /* temporal decay of the cache per frame */
    float variance_norm;            /* core.hpp:109 (VARIANCE view and rank.comp variance scale) */
    uint32_t flags;                 /* VE_FRAME_* */
    /* importance-aware scheduling (VE_FRAME_SCHEDULED), core.hpp:95-112 */
    float weight_pixels;            /* 0.1 */
    float weight_variance;          /* 0.9 */
    float pixels_norm;              /* 100 */
    float top_fraction;             /* 0.30: voxels given 2 paths */
    float mid_fraction;             /* 0.40: voxels given 1 path */
    uint32_t min_samples;           /* 1: paths of the remaining voxels */
    uint32_t shading_budget;        /* 131072: cap on paths per frame */
    /* emissive NEE (VE_FRAME_EMISSIVE), ReSTIR DI knobs of core.hpp:138-144 */
    uint32_t restir;                  /* VE_RESTIR_* bits; all three by default */
    uint32_t restir_m;                /* 4: initial RIS candidates (<= 64) */
    uint32_t restir_spatial_neighbors;/* 1 (at most 6 are used) */
    uint32_t restir_max_m;            /* 24: history cap on reuse */
    float restir_spatial_radius;      /* 2.75: neighbour offset in voxels */
    /* dual-channel lBuffer (VE_FRAME_LBUFFER), core.hpp:93-104, 150-157 */
    uint32_t time;                    /* the caller's clock for the stale reset (the reference: 1/100 s) */
    uint32_t update_time;             /* a slot older than this is reset on its next deposit */
    uint32_t disable_stale_reset;
    uint32_t sample_cap_direct;       /* 16: the direct channel halves at this count */
    uint32_t sample_cap_indirect;     /* 64 */
    float firefly_k;                  /* 1: a sample above k x the running mean is scaled down */
    float firefly_floor;              /* 255: lower bound of that threshold (quantised units) */
    /* split frames (VE_FRAME_SPLIT): this rank's band of rows */
    uint32_t row_begin, row_end;
} ve_frame_config;

#define VE_RESTIR_ENABLE 1u   /* ReSTIR DI at bounce 0 (else single-pick RIS there too) */
#define VE_RESTIR_TEMPORAL 2u /* reuse the voxel's reservoir from earlier frames */
#define VE_RESTIR_SPATIAL 4u  /* reuse neighbour voxels' reservoirs */

/* One render request: scene, Camera::UBO (camera.hpp:24-29: position,
 * cameraPlane, cameraPlaneRight, cameraPlaneUp as 4 x vec4) and frame knobs. */
typedef struct ve_view {
    int32_t scene_id;
    float camera[16];
    ve_frame_config frame;
} ve_view;

/* Outputs of one view (host pointers; NULL = not requested).  gbuffer is the
 * GBuffer image (generate_primary.comp:68-82) with the hit-node index in the
 * reserved .z lane; rgb is the AvgPass output (avgPass.texture); mapped is
 * the RenderPass ACES output (final.frag:11-18). */
typedef struct ve_frame_outputs {
    uint32_t* gbuffer;  /* 4 x u32 per pixel {checks, material, hit node, vid} */
    uint32_t* voxel_id; /* 1 x u32 per pixel: voxelKey + 1, 0 on miss */
    uint32_t* hit_node; /* 1 x u32 per pixel: node slot of the hit leaf, 0 on miss */
    float* rgb;         /* 3 x f32 per pixel */
    float* mapped;      /* 3 x f32 per pixel */
    float* path_rgb;    /* 3 x f32 per path (pixel * spp + sample); VE_FRAME_PATH_RGB;
                           zero for pixels without a primary hit (no path).  With
                           VE_FRAME_SCHEDULED: one per shade-list entry, room for
                           min(shading_budget, 2 * width * height) paths */
    uint8_t* mapped8;   /* 4 x u8 per pixel: the displayed image, FragColor =
                           (mapped, 1) as an RGBA8 framebuffer stores it (final.frag:15-18:
                           clamp to [0, 1], x 255, round to nearest) */
} ve_frame_outputs;

/* FrameStats (src/renderer/core.hpp:164-185) and the profiler's stage
 * timings (src/renderer/profiler.hpp:43-70), from device counters and CUDA
 * events of the last ve_render / ve_render_batch call. */
typedef struct ve_frame_stats {
    uint64_t rays_primary, rays_bounce, rays_shadow;
    uint64_t fetch_nodes; /* node words read by every DDA (VE_FRAME_COUNT_FETCH) */
    uint64_t paths, deposits, deposits_dropped;
    uint64_t dda_steps;   /* DDA outer iterations (VE_FRAME_COUNT_FETCH) */
    uint64_t fetch_nodes_trace, dda_steps_trace; /* the bounce/shadow trace kernel alone */
    uint64_t h2d_bytes, d2h_bytes;               /* bytes the call(s) copied host<->device */
    uint64_t frames;                             /* render calls covered */
    float ms_total, ms_primary, ms_trace, ms_shade, ms_resolve, ms_decay; /* VE_FRAME_TIMING */
    uint32_t trace_launches, kernel_launches;
    uint64_t cache_capacity;
    uint64_t nrc_queries;         /* paths ended by the learned cache */
    uint64_t nrc_hash_terminated; /* paths ended by the hashed per-voxel cache */
    uint64_t nrc_samples;         /* training samples recorded */
    uint64_t scheduled_voxels;    /* VE_FRAME_SCHEDULED: distinct visible voxels */
    uint64_t scheduled_paths;     /* VE_FRAME_SCHEDULED: shade-list entries (paths) */
    float ms_learned;             /* learned-cache inference + training (VE_FRAME_TIMING) */
    uint32_t reserved;
    uint64_t emissive_lights;     /* VE_FRAME_EMISSIVE: registered lights after the call */
    uint64_t nee_emissive;        /* VE_FRAME_EMISSIVE: NEE shadow rays toward lights */
    uint64_t restir_commits;      /* VE_FRAME_EMISSIVE: voxel reservoirs stored */
    uint64_t shadow_shared;       /* sun shadow rays counted in rays_shadow but not traced: a pixel's
                                     samples share their first shading step's shadow ray (the same
                                     origin and direction), traced once, by sample 0 */
} ve_frame_stats;

typedef struct ve_ctx ve_ctx;
typedef struct ve_octree_cpu ve_octree_cpu;
typedef struct ve_octree ve_octree;
typedef struct ve_words ve_words;

const char* ve_version(void);
const char* ve_last_error(void);

/* ======================================================================
 * Host scene layer
 * ==================================================================== */

/* OctreeCPU (src/octree_cpu.hpp:27-37): ctor, insert, remove, lookup,
 * insertBox, insertSphere, raycast. */
int ve_octree_cpu_create(uint32_t depth, ve_octree_cpu** out);
int ve_octree_cpu_destroy(ve_octree_cpu* t);
int ve_octree_cpu_insert(ve_octree_cpu* t, uint32_t x, uint32_t y, uint32_t z, uint32_t material);
int ve_octree_cpu_insert_many(ve_octree_cpu* t, const uint32_t* xyzm, uint64_t n);
int ve_octree_cpu_remove(ve_octree_cpu* t, uint32_t x, uint32_t y, uint32_t z);
/* material of the leaf at (x,y,z), or -1 when absent (OctreeCPU::lookup) */
int ve_octree_cpu_lookup(const ve_octree_cpu* t, uint32_t x, uint32_t y, uint32_t z, int64_t* material);
int ve_octree_cpu_insert_box(ve_octree_cpu* t, const uint32_t mn[3], const uint32_t mx[3], uint32_t material);
int ve_octree_cpu_insert_sphere(ve_octree_cpu* t, const float centre[3], float radius, uint32_t material);
int ve_octree_cpu_raycast(const ve_octree_cpu* t, const float origin[3], const float dir[3], uint32_t max_steps,
                          int* hit, uint32_t pos[3]);

/* Octree (src/renderer/octree.hpp:45-59): the node array in the reference
 * layout.  ve_octree_words returns `capacity` words (valid until the next
 * set / apply_edits). */
int ve_octree_create(uint32_t depth, ve_octree** out);
int ve_octree_destroy(ve_octree* o);
int ve_octree_set(ve_octree* o, ve_octree_cpu* cpu);                     /* Octree::set */
int ve_octree_apply_edits(ve_octree* o, ve_octree_cpu* cpu, uint32_t* changed_slots, uint64_t cap,
                          uint64_t* n_changed);                           /* Octree::applyEdits */
/* the changed slots of the last ve_octree_apply_edits (valid until the next call) */
int ve_octree_last_changed(const ve_octree* o, const uint32_t** slots, uint64_t* n);
int ve_octree_find_gpu_slot(const ve_octree* o, ve_octree_cpu* cpu, uint32_t x, uint32_t y, uint32_t z,
                            uint32_t* slot);                              /* Octree::findGpuSlot */
int ve_octree_info(const ve_octree* o, uint32_t* size, uint32_t* capacity, uint32_t* num_voxels);
int ve_octree_words(const ve_octree* o, const uint32_t** words, uint64_t* n);

/* Seeded value-noise terrain scenes (benchmark inputs; no reference
 * counterpart: the reference's demo scene is built in voxelengine.cpp:129-144).
 * ve_terrain_build emits the words of OctreeCPU::insert + Octree::set in
 * parallel without pointer nodes. */
int ve_terrain_build(uint32_t depth, uint32_t variant, uint64_t seed, uint32_t threads, ve_words** out,
                     uint64_t* n_voxels);
int ve_words_data(const ve_words* w, const uint32_t** data, uint64_t* n);
int ve_words_free(ve_words* w);
int ve_terrain_voxels(uint32_t depth, uint32_t variant, uint64_t seed, uint32_t* xyzm, uint64_t cap, uint64_t* n);
int ve_terrain_materials(uint64_t seed, void* out_128_std140_entries);

/* Camera::UpdateUBO (src/renderer/camera.cpp:39-50) */
int ve_camera_ubo(const float pos[3], const float dir[3], float fov_deg, float aspect, float ubo[16]);

/* ======================================================================
 * Device renderer
 * ==================================================================== */

/* Renderer::Renderer (src/renderer/renderer.hpp:11-12) / ~Renderer */
int ve_ctx_create(const ve_renderer_config* cfg, ve_ctx** out);
int ve_ctx_destroy(ve_ctx* ctx);
/* the context's cudaStream_t, for callers that time or order work on it */
int ve_ctx_stream(ve_ctx* ctx, void** stream);
int ve_ctx_synchronize(ve_ctx* ctx);
/* Orders work enqueued on the context's stream after this call behind every
 * frame rendered so far (VE_CFG_PIPELINE runs some on a second stream). */
int ve_ctx_join(ve_ctx* ctx);

/* Octree::set upload (octree.cpp:157-159 glBufferData of Octree::data):
 * `words` verbatim in the reference layout.  Unless VE_SCENE_KEEP_NORMALS,
 * a device pass fills every leaf's normal field (3x3x3 occupancy gradient). */
int ve_scene_upload(ve_ctx* ctx, const uint32_t* words, uint64_t n_words, uint32_t depth, uint32_t flags,
                    int32_t* scene_id);
/* GPU bulk build (no counterpart in the reference): the node words that
 * OctreeCPU::insert of every voxel followed by Octree::set produce, built on
 * the device from n host rows (x, y, z, material 1..127) — a repeated
 * position keeps its last row — and uploaded as a scene like
 * ve_scene_upload.  *n_words (may be NULL) receives the array size. */
int ve_scene_build(ve_ctx* ctx, const uint32_t* xyzm, uint64_t n, uint32_t depth, uint32_t flags,
                   int32_t* scene_id, uint64_t* n_words);
int ve_scene_release(ve_ctx* ctx, int32_t scene_id);
/* Targeted refresh after an edit, the counterpart of the reference's
 * findGpuSlot-driven invalidation (octree.cpp:317-341): for every voxel in
 * the 3x3x3 neighbourhood of each of the n edited positions (x, y, z), the
 * leaf normal field is recomputed (same values as the full pass) and, unless
 * VE_REFRESH_KEEP_CACHE, the voxel's radiance-cache entry is cleared.  Use
 * after ve_scene_apply_edits(..., VE_SCENE_KEEP_NORMALS) in place of the full
 * normal pass. */
#define VE_REFRESH_KEEP_CACHE 1u
int ve_scene_refresh(ve_ctx* ctx, int32_t scene_id, const uint32_t* xyz, uint64_t n, uint32_t flags);
/* Octree::applyEdits upload (octree.cpp:228-314 UpdateNode): scatter
 * words[i] to slots[i]; normals of affected leaves are recomputed unless
 * VE_SCENE_KEEP_NORMALS.  The scene's radiance cache is kept. */
int ve_scene_apply_edits(ve_ctx* ctx, int32_t scene_id, const uint32_t* slots, const uint32_t* words, uint64_t n,
                         uint32_t flags);
/* Per-voxel normal mode of a scene (replaces the normalPrecision uniform of
 * the reference's normal pass, src/renderer/core.hpp:88 and
 * src/shd/normal.comp:55-95).  radius 0: the 3x3x3 occupancy gradient (the
 * default at upload).  radius R >= 1: the reference's computeRefinedNormal —
 * the offsets of the empty neighbours with 0 < |d|^2 <= R^2 around the
 * voxel's even-aligned corner (normal.comp:147-152), out-of-volume neighbours
 * empty, normalized ((0,1,0) for a zero sum), 10-10-10 packed
 * (packNormalAccum); the scene keeps the sorted table of its distinct codes
 * and each leaf's normal field (bits 8-30, bit 31 clear) holds its code's
 * index + 1.  Recomputes every leaf now; later full normal passes
 * (ve_scene_apply_edits without VE_SCENE_KEEP_NORMALS) keep the mode, and
 * ve_scene_refresh is refused (VE_ERR_STATE) for ball-mode scenes.  Scenes of
 * depth <= 11; VE_ERR_INVALID for radius > VE_NORMAL_BALL_MAX_RADIUS. */
#define VE_NORMAL_BALL_MAX_RADIUS 16u
int ve_scene_normal_mode(ve_ctx* ctx, int32_t scene_id, uint32_t radius);
int ve_scene_download(ve_ctx* ctx, int32_t scene_id, uint32_t* out, uint64_t cap, uint64_t* n_words);

/* A batch of independent rays through the device DDA that the frame kernels
 * run (Raycast / RaycastCounted, src/shd/internal.glsl:297-400; the GPU
 * counterpart of OctreeCPU::raycast, src/octree_cpu.cpp:128-215, for
 * picking and for checking the traversal ray by ray).  origins, dirs: 3 f32
 * per ray, host memory; out: 8 u32 per ray {status (0 hit, 1 left the
 * volume, 2 out of controlchecks), hit node slot, material, x, y, z, node
 * size, checks}.  flags: VE_RAYCAST_FULL_WALK descends every octree level
 * per step instead of starting from the scene's top table.  Synchronous. */
#define VE_RAYCAST_FULL_WALK 1u
int ve_raycast_batch(ve_ctx* ctx, int32_t scene_id, const float* origins, const float* dirs, uint64_t n,
                     uint32_t controlchecks, uint32_t flags, uint32_t* out);
/* device bytes held by a scene: node array, radiance cache and top table
 * (4 B per cell of the grid one level above the leaves, for depths up to 10:
 * 512 MiB at depth 10 and deeper) */
int ve_scene_footprint(ve_ctx* ctx, int32_t scene_id, uint64_t* bytes);
/* The box bounce rays are clipped to (no reference counterpart: a bound the
 * trace derives from the top table).  A bounce ray whose escape and timeout
 * shade alike ends, as escaped, once it has left the box of the top-table
 * cells that hold voxels, widened by one voxel: it can hit nothing after
 * that.  *bounded = 0 (lo/hi = -/+1e30) when no box applies: scenes without
 * a top table (depth < 3), deeper than 12, or whose faces {x, y or z = 2^D}
 * (inside the DDA's bounds test, read through root words 1..7) hold a
 * voxel.  Recomputed by every upload, build and edit. */
int ve_scene_clip_box(ve_ctx* ctx, int32_t scene_id, float lo[3], float hi[3], uint32_t* bounded);

/* MaterialPool UBO (src/renderer/material.cpp:17-49): n entries of 64 B
 * (std140 Material), index 0 reserved. */
int ve_set_materials(ve_ctx* ctx, const void* entries, uint32_t n);

/* Radiance cache of a scene (the lBuffer replacement): clear, and dump of
 * occupied entries: vids, exact deposit counts, and 5 floats per entry
 * {decayed weight, r, g, b, luma^2} sums. */
int ve_cache_reset(ve_ctx* ctx, int32_t scene_id);
int ve_cache_dump(ve_ctx* ctx, int32_t scene_id, uint32_t* vids, uint32_t* counts, float* values, uint64_t cap,
                  uint64_t* n);
/* The scene's dual-channel lBuffer (VE_FRAME_LBUFFER frames): every occupied
 * slot as 14 u32 {row, slot, vid, dir count, dir r, g, b, dir L^2, ind count,
 * ind r, g, b, ind L^2, last time} in (row, slot) order; `n` = the occupied
 * slots (records written: min(n, cap)).  Nothing before the first lBuffer
 * frame. */
int ve_lbuffer_dump(ve_ctx* ctx, int32_t scene_id, uint32_t* out, uint64_t cap, uint64_t* n);

/* Renderer::run (src/renderer/renderer.hpp:13, renderer.cpp:282-712): one
 * frame of one view.  Returns after the host outputs are written; with all
 * output pointers NULL it only enqueues the work on the context stream. */
int ve_render(ve_ctx* ctx, const ve_view* view, ve_frame_outputs* out);
/* Several views (any scenes, resolutions, spp, bounces) as one wavefront
 * batch: one primary pass over all views, one trace and one shade pass per
 * bounce depth for all their paths, one resolve pass. `outs` may be NULL. */
int ve_render_batch(ve_ctx* ctx, const ve_view* views, uint32_t n_views, ve_frame_outputs* outs);
/* Split frames (one frame of one view over several GPUs, each rendering a
 * band of rows; the multi-GPU form of Renderer::run for frames too large
 * for one device).  A rank renders its band with VE_FRAME_SPLIT (ve_render:
 * primary rays of the band and of max(reconstruction_radius, 1) rows on
 * either side, paths of the band's pixels only; the scene's cache is
 * decayed, the frame's deposits go to a per-frame table; no AvgPass, and
 * rgb / mapped outputs must be NULL).  Then every rank:
 *   ve_split_export  the per-frame table as records (device memory),
 *   (all-gather of the records across ranks: NCCL over NVLink),
 *   ve_split_merge   every rank's records, in rank order, into the cache,
 *   ve_split_resolve the AvgPass of the band.
 * All ranks merge the same records in the same order, so their caches stay
 * identical; the merged cache holds the counts of the unsplit frame and its
 * sums up to float rounding.  A record is 8 x 32-bit words {vid, count,
 * luma^2, r, g, b, weight, 0} (32 B). */
typedef struct ve_split_record {
    uint32_t vid, count;
    float l2, r, g, b, w;
    uint32_t reserved;
} ve_split_record;
/* Records of the last VE_FRAME_SPLIT frame of `scene_id` into device memory
 * `dev_out` (room for `cap`); `n` = records in the frame (written: min(n,
 * cap)).  A frame's records are exported once: the export empties the
 * per-frame table.  Synchronous. */
int ve_split_export(ve_ctx* ctx, int32_t scene_id, void* dev_out, uint64_t cap, uint64_t* n);
/* Adds `n_parts` record arrays (device memory; part k starts at record
 * k * stride and holds counts[k] records) into the scene's cache, part 0
 * first.  `dropped` (may be NULL): records whose voxel found no cache entry.
 * Synchronous. */
int ve_split_merge(ve_ctx* ctx, int32_t scene_id, const void* dev_parts, const uint64_t* counts, uint32_t n_parts,
                   uint64_t stride, uint64_t* dropped);
/* The AvgPass (resolve.comp) of the band of `view` (the view of the last
 * VE_FRAME_SPLIT render) from the merged cache; the outputs' rows
 * [row_begin, row_end) are written (host pointers to full-size images). */
int ve_split_resolve(ve_ctx* ctx, const ve_view* view, ve_frame_outputs* out);

/* Launch shape of the persistent bounce kernels: resident blocks per SM of
 * the trace and shade kernels (0 = occupancy maximum) and the number of idle
 * lanes at which a trace warp refills itself with new rays (0 = default, 20). */
typedef struct ve_launch_config {
    uint32_t trace_blocks_per_sm;
    uint32_t shade_blocks_per_sm;
    uint32_t refill_threshold;
    uint32_t reserved;
} ve_launch_config;
int ve_get_launch_config(ve_ctx* ctx, ve_launch_config* cfg);
int ve_set_launch_config(ve_ctx* ctx, const ve_launch_config* cfg);
/* Autotuner (no reference counterpart): renders the given views with
 * candidate launch shapes (coordinate descent over trace blocks/SM, shade
 * blocks/SM, refill threshold; `frames_per_trial` timed frames each), keeps
 * the fastest in the context and returns it.  The trial frames deposit into
 * the scenes' radiance caches like any render. */
int ve_autotune(ve_ctx* ctx, const ve_view* views, uint32_t n_views, uint32_t frames_per_trial,
                ve_launch_config* best);

/* stats of the last render call (synchronises the context stream) */
int ve_get_stats(ve_ctx* ctx, ve_frame_stats* stats);
/* stats summed over every render call since ve_reset_total_stats (device
 * counters accumulate on the stream: no host synchronisation per frame) */
int ve_get_total_stats(ve_ctx* ctx, ve_frame_stats* stats);
int ve_reset_total_stats(ve_ctx* ctx);

/* ======================================================================
 * Render server: continuous batching (no reference counterpart; the
 * reference renders one interactive view per Renderer::run)
 * ==================================================================== */

/* Requests are admitted while their framebuffer (pixel_capacity pool) and
 * path-state (path_capacity pool) ranges fit — the per-request part of the
 * HBM budget; scenes and radiance caches stay resident — and join the
 * in-flight wavefront at the next bounce pass.  Admission takes queued
 * requests in arrival order and passes over one that does not fit yet, unless
 * it has waited longer than max_bypass_ms: then nothing behind it is admitted
 * until it fits (the pools drain for it).  Each step starts the primary pass
 * of at most step_path_budget paths: a larger request's tiles are spread over
 * several steps, so no step grows long enough to hold up the small requests
 * in flight.  VE_SERVER_FIFO restores strict first-come-first-served
 * admission with each request's whole primary pass in one step.  The server
 * owns the context's stream while it exists.  Requests render the plain
 * method: the PATH_RGB, SCHEDULED, EMISSIVE, LBUFFER, SPLIT, LEARNED, TRAIN
 * and TERMINATE_HASH frame flags are ignored. */
#define VE_SERVER_FIFO 1u
typedef struct ve_server ve_server;
typedef struct ve_server_config {
    uint64_t pixel_capacity;   /* pooled pixels: GBuffer + outputs, 48 B each */
    uint64_t path_capacity;    /* pooled path states, 152 B each (below 2^30) */
    uint32_t max_requests;     /* view slots (requests on the GPU at once) */
    uint32_t flags;            /* VE_SERVER_FIFO */
    uint64_t step_path_budget; /* paths whose primary pass one step may start (0: 2^23) */
    uint32_t max_bypass_ms;    /* how long a request that does not fit may be passed over (0: 50 ms) */
    uint32_t reserved;
} ve_server_config;
typedef struct ve_request_info {
    uint64_t request_id;
    double submit_s, admit_s, done_s; /* steady-clock seconds */
    uint64_t pixels, paths;
} ve_request_info;
typedef struct ve_server_stats {
    uint64_t completed, admitted, queued, in_flight, max_in_flight, steps;
    uint64_t pool_bytes, scene_bytes;
    uint64_t rays; /* primary + bounce + shadow rays traced since creation */
} ve_server_stats;
int ve_server_create(ve_ctx* ctx, const ve_server_config* cfg, ve_server** out);
/* voxel_id_out (1 x u32 per pixel) and rgb_out (3 x f32 per pixel) may be NULL;
 * they must stay valid until ve_server_wait returns for this request */
int ve_server_submit(ve_server* s, const ve_view* view, uint32_t* voxel_id_out, float* rgb_out,
                     uint64_t* request_id);
/* waits for a request (VE_ERR_TIMEOUT when not done within timeout_ms), then
 * forgets it */
int ve_server_wait(ve_server* s, uint64_t request_id, uint32_t timeout_ms, ve_request_info* info);
int ve_server_get_stats(ve_server* s, ve_server_stats* stats);
/* finishes queued and in-flight requests, then stops the worker */
int ve_server_destroy(ve_server* s);

/* ======================================================================
 * Learned radiance cache (no counterpart in the reference)
 *
 * A multi-resolution hash-grid encoding (16 levels x 2 fp16 features) of the
 * voxel position, the octahedral shading normal and the octahedral view
 * direction feed a 4 x 64 ReLU MLP with a 3-channel output, evaluated and
 * trained with bf16 tensor-core kernels (f32 accumulation, Adam).  Attached to
 * a scene (ve_scene_set_nrc), it terminates paths at their second vertex in
 * frames rendered with VE_FRAME_LEARNED and trains online on the paths of
 * frames rendered with VE_FRAME_TRAIN.
 * ==================================================================== */
typedef struct ve_nrc ve_nrc;
typedef struct ve_nrc_config {
    uint32_t log2_table;      /* entries per hash-grid level, log2 (19) */
    uint32_t base_resolution; /* coarsest grid resolution (16) */
    uint32_t max_resolution;  /* finest grid resolution (2048) */
    uint32_t train_samples;   /* training samples per frame (65536) */
    float learning_rate;      /* Adam step size (1e-2) */
    float beta1, beta2, eps;  /* Adam moments (0.9, 0.99, 1e-8) */
    float fallback_threshold; /* per-cell validation error above which the hash cache answers (0.1) */
    uint32_t flags;
    uint64_t seed;            /* parameter initialisation */
} ve_nrc_config;
typedef struct ve_nrc_input {
    float pos[3];        /* voxel centre / scene extent, in [0,1)^3 */
    uint32_t reserved;
    float normal_oct[2]; /* octahedral shading normal */
    float view_oct[2];   /* octahedral direction toward the previous path vertex */
} ve_nrc_input;
int ve_nrc_create(ve_ctx* ctx, const ve_nrc_config* cfg, ve_nrc** out);
int ve_nrc_destroy(ve_nrc* nrc);
/* weights: 5 x 64 x 64 f32 (layer 5 uses rows 0-2); table: 16 x 2^log2_table x 2 f32 */
int ve_nrc_param_counts(const ve_nrc* nrc, uint64_t* n_weights, uint64_t* n_table);
int ve_nrc_get_params(ve_nrc* nrc, float* weights, float* table);
/* replaces the parameters and restarts the optimiser */
int ve_nrc_set_params(ve_nrc* nrc, const float* weights, const float* table);
/* rgb: n x 3 predictions */
int ve_nrc_infer(ve_nrc* nrc, const ve_nrc_input* in, uint32_t n, float* rgb);
/* gradients of the mean relative L2 loss over the n samples, without an update */
int ve_nrc_gradients(ve_nrc* nrc, const ve_nrc_input* in, const float* target, uint32_t n, float* weight_grad,
                     float* table_grad, float* loss);
/* one Adam step on the n samples; loss before the step */
int ve_nrc_train(ve_nrc* nrc, const ve_nrc_input* in, const float* target, uint32_t n, float* loss);
/* mean training loss of the last training step (learned frames or
 * ve_nrc_train), its sample count, and the number of steps taken */
int ve_nrc_stats(ve_nrc* nrc, float* loss, uint64_t* samples, uint64_t* steps);
/* attaches (or, with NULL, detaches) a learned cache to a scene */
int ve_scene_set_nrc(ve_ctx* ctx, int scene_id, ve_nrc* nrc);

/* ======================================================================
 * Allocation-free entry point (no counterpart in the reference)
 * ==================================================================== */

/* Fills the normal field of every leaf of a node array that already lives in
 * device memory (the same 3x3x3 occupancy-gradient pass ve_scene_upload runs),
 * without allocating anything.  It exists for callers that may not call
 * cudaMalloc: hosts that own the whole device-memory budget (an engine's or a
 * service's arena) and forbid libraries from allocating behind them, and
 * latency-critical threads that cannot afford cudaMalloc/cudaFree stalling the
 * device.  The caller passes the device node array; the work is enqueued on
 * `stream` (a cudaStream_t, NULL = default stream) and is complete when the
 * stream reaches it.
 *
 * Scratch: a fixed file-scope device array of VE_NOALLOC_SCRATCH_BYTES
 * (frontiers + occupancy bitmask), present on every GPU that loads the
 * library until the process exits, which limits the scene to depth <= 7
 * (VE_ERR_CAPACITY beyond).  The first call on a device looks up that array's
 * device address with the device current, and so does the first call after
 * the current context changed (cudaDeviceReset, or another context made
 * current); make those calls before any stream capture.  All calls share the
 * one array: calls that overlap on the GPU (on different streams, or from
 * several threads) race on it.  A well-formed depth-7 array never outgrows
 * the scratch; a malformed one (blocks that point back up the tree) can, and
 * then the cells beyond the scratch are skipped: the call still returns
 * VE_OK with only some normals filled. */
#define VE_NOALLOC_MAX_DEPTH 7
#define VE_NOALLOC_SCRATCH_BYTES (256u + 2u * (1u << 18) * 8u + (1u << 21) / 8u)
int ve_fill_normals_noalloc(uint32_t* device_words, uint64_t n_words, uint32_t depth, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* VE_H */
