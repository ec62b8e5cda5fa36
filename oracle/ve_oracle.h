// ve_oracle.h — TEST INFRASTRUCTURE ONLY (the checker, never the product).
//
// Scalar C++ restatement of the reference's ray pipeline
// (AnghelusAndrei/VoxelEngine3.0): octree DDA (src/shd/internal.glsl:297-400),
// voxel keys (internal.glsl:263-291), the Halton RNG (internal.glsl:57-98)
// seeded as src/shd/emit.comp:171-174, the bounce/shade loop
// (src/shd/shade.comp:543-575, 838-908), the accumulation (AccumPass) and the
// averaging (AvgPass, src/shd/resolve.comp:109-148, 193-261) with the
// substitutions of the plain benchmark method: directional sun + constant sky,
// FP decayed per-voxel radiance cache, per-leaf 3x3x3 occupancy-gradient
// normals, per-pixel spp.  Only tests/, __graft_entry__.smoke() and bench.py's
// CPU-baseline leg may load this library.
#pragma once
#include <cstdint>

extern "C" {

// Frame parameters (same field order as the product's ve_frame_config).
struct ov_frame_params {
    uint32_t width, height;
    uint32_t spp;
    uint32_t bounces;
    uint32_t primary_controlchecks;
    uint32_t bounce_controlchecks;
    uint32_t reconstruction_radius;
    uint32_t render_type;
    uint32_t frame_index;
    float sun_dir[3];
    float sun_intensity;
    float sky[3];
    float decay;
    float variance_norm;
    uint32_t flags;
    /* importance-aware scheduling (flags & 64), core.hpp:95-112 */
    float weight_pixels, weight_variance, pixels_norm, top_fraction, mid_fraction;
    uint32_t min_samples, shading_budget;
    /* emissive NEE (flags & 128), core.hpp:138-144 */
    uint32_t restir, restir_m, restir_spatial_neighbors, restir_max_m;
    float restir_spatial_radius;
    /* dual-channel lBuffer (flags & 256), core.hpp:93-104, 150-157 */
    uint32_t time, update_time, disable_stale_reset, sample_cap_direct, sample_cap_indirect;
    float firefly_k, firefly_floor;
};

struct ov_stats {
    uint64_t rays_primary, rays_bounce, rays_shadow;
    uint64_t fetch_restart;   // node words read by restart-from-root descent
    uint64_t fetch_min;       // distinct (level, node) words per ray (summed)
    uint64_t paths, deposits;
    uint64_t steps;           // DDA outer iterations (all rays)
    uint64_t scheduled_voxels, scheduled_paths;  // scheduled frames
    uint64_t emissive_lights, nee_emissive, restir_commits;  // emissive frames
    uint64_t shadow_shared;   // first shadow rays of a pixel's later samples (sample 0's walk)
};

}  // extern "C"
