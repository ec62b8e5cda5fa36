// lbuffer.cuh — the reference's dual-channel lBuffer AccumPass
// (src/shd/shade.comp:96-257 depositSampleDual; src/shd/resolve.comp:109-148
// lookupVoxelAvg; src/shd/rank.comp:66-87 lookupIndirectVariance) for
// VE_FRAME_LBUFFER.
//
// A row of kLbSlots slots of kLbStride words per hash row vid % (W-1) + 1:
//   +0 vid   +1 dir count  +2..4 dir r,g,b sums  +5 dir L^2 sum
//            +6 ind count  +7..9 ind r,g,b sums  +10 ind L^2 sum  +11 last time
// with samples quantised as uint(clamp(c, 0, 1024) * 255), per-channel
// halving at the sample caps, the firefly clamp against the running mean,
// the stale reset after `update_time` and least-recently-used replacement.
//
// Determinism: the reference's deposits race on the slots' atomics, so the
// result depends on the arrival order.  Here a frame's deposits are
// collected, ordered by (row, path slot) and applied row by row in that
// order — the same operations the reference performs, in one fixed order
// that the oracle repeats.
#pragma once
#include <cstdint>

namespace ve {
namespace dev {

constexpr uint32_t kLbWidth = 32768;  // rows (the reference: GL_MAX_TEXTURE_SIZE)
constexpr uint32_t kLbSlots = 32;     // LBUFFER_SLOTS (renderer.hpp:90)
constexpr uint32_t kLbStride = 12;    // lBufferStride (wavefront.glsl:204)
constexpr uint32_t kLbRowWords = kLbSlots * kLbStride;

struct LbParams {
    uint32_t time, update_time, disable_stale, cap_dir, cap_ind;
    float firefly_k, firefly_floor;
};

// A path's deposit: clamped direct and indirect radiance.
struct LbRec {
    uint32_t vid, slot;
    float d[3], e[3];
};
static_assert(sizeof(LbRec) == 32, "deposit record");

__host__ __device__ __forceinline__ uint32_t lb_row(uint32_t vid) { return vid % (kLbWidth - 1u) + 1u; }

// packRgbL2 (shade.comp:154-160); GLSL uint arithmetic wraps.
__device__ __forceinline__ void lb_pack(const float c[3], uint32_t out[4]) {
    for (int k = 0; k < 3; k++) out[k] = uint32_t(gclamp(c[k], 0.0f, 1024.0f) * 255.0f);
    const uint32_t L = (out[0] + out[1] + out[2]) / 3u;
    out[3] = L * L;
}

__device__ __forceinline__ void lb_reset(uint32_t* s, uint32_t vid, const uint32_t d[4], const uint32_t e[4],
                                         uint32_t time) {  // resetLSlotDual
    s[0] = vid;
    s[1] = 1u; s[2] = d[0]; s[3] = d[1]; s[4] = d[2]; s[5] = d[3];
    s[6] = 1u; s[7] = e[0]; s[8] = e[1]; s[9] = e[2]; s[10] = e[3];
    s[11] = time;
}

__device__ __forceinline__ void lb_firefly(const uint32_t* s, uint32_t c[4], const LbParams& P) {
    const uint32_t n = s[0];  // count (s points at the channel's count word)
    if (n > 4u) {
        const float meanL = float(s[1] + s[2] + s[3]) / float(3u * n);
        const float sampleL = float(c[0] + c[1] + c[2]) / 3.0f;
        const float thresh = gmax(meanL * P.firefly_k, P.firefly_floor);
        if (sampleL > thresh) {
            const float scale = thresh / sampleL;
            c[0] = uint32_t(float(c[0]) * scale);
            c[1] = uint32_t(float(c[1]) * scale);
            c[2] = uint32_t(float(c[2]) * scale);
            const uint32_t L = (c[0] + c[1] + c[2]) / 3u;
            c[3] = L * L;
        }
    }
}

// A deposit into the slot that holds `vid` (shade.comp:184-254): the stale
// reset, the per-channel halving at the caps, the firefly clamp, the sums.
__device__ __forceinline__ void lb_update(uint32_t* s, uint32_t vid, uint32_t d[4], uint32_t e[4],
                                          const LbParams& P) {
    const uint32_t t = s[11];
    if (!P.disable_stale && t != 0u && t + P.update_time < P.time) {
        lb_reset(s, vid, d, e, P.time);
        return;
    }
    if (s[1] >= P.cap_dir)
        for (int k = 1; k <= 5; k++) s[k] >>= 1;
    if (s[6] >= P.cap_ind)
        for (int k = 6; k <= 10; k++) s[k] >>= 1;
    lb_firefly(s + 1, d, P);
    lb_firefly(s + 6, e, P);
    s[1] += 1u; s[2] += d[0]; s[3] += d[1]; s[4] += d[2]; s[5] += d[3];
    s[6] += 1u; s[7] += e[0]; s[8] += e[1]; s[9] += e[2]; s[10] += e[3];
    s[11] = P.time;
}

// depositSampleDual (shade.comp:162-257) on a whole row, sequentially.
__device__ __forceinline__ void lb_deposit(uint32_t* row, uint32_t vid, const float dir[3], const float ind[3],
                                           const LbParams& P) {
    uint32_t d[4], e[4];
    lb_pack(dir, d);
    lb_pack(ind, e);
    uint32_t cand_t = 0xFFFFFFFFu, cand_i = 0u;
    for (uint32_t i = 0; i < kLbSlots; i++) {
        uint32_t* s = row + i * kLbStride;
        if (s[0] == 0u) s[0] = vid;  // claim an empty slot
        if (s[0] != vid) {
            if (s[11] < cand_t) {
                cand_t = s[11];
                cand_i = i;
            }
            continue;
        }
        lb_update(s, vid, d, e, P);
        return;
    }
    if (cand_t != 0xFFFFFFFFu) lb_reset(row + cand_i * kLbStride, vid, d, e, P.time);
}

// lookupVoxelAvg (resolve.comp:109-148): direct mean + indirect mean, the
// combined count, the indirect variance on the [0, 1] scale.
__device__ __forceinline__ bool lb_lookup(const uint32_t* lb, uint32_t vid, f3& rgb, uint32_t& count, float& var) {
    rgb = mk(0.0f, 0.0f, 0.0f);
    count = 0u;
    var = 0.0f;
    if (vid == 0u) return false;
    const uint32_t* row = lb + size_t(lb_row(vid)) * kLbRowWords;
    for (uint32_t i = 0; i < kLbSlots; i++) {
        const uint32_t* s = row + i * kLbStride;
        if (s[0] != vid) continue;
        const uint32_t dc = s[1], ic = s[6];
        count = dc + ic;
        if (count == 0u) return true;
        f3 da = mk(0.0f, 0.0f, 0.0f), ia = da;
        if (dc > 0u) {
            const float inv = 1.0f / float(dc);
            da = mk(float(s[2]) * inv / 255.0f, float(s[3]) * inv / 255.0f, float(s[4]) * inv / 255.0f);
        }
        if (ic > 0u) {
            const float inv = 1.0f / float(ic);
            ia = mk(float(s[7]) * inv / 255.0f, float(s[8]) * inv / 255.0f, float(s[9]) * inv / 255.0f);
            const float meanL = float(s[7] + s[8] + s[9]) * inv / 3.0f;
            var = gmax(float(s[10]) * inv - meanL * meanL, 0.0f) / (255.0f * 255.0f);
        }
        rgb = add(da, ia);
        return true;
    }
    return false;
}

// lookupIndirectVariance (rank.comp:66-87), raw quantised units.
__device__ __forceinline__ float lb_indirect_variance(const uint32_t* lb, uint32_t vid) {
    const uint32_t* row = lb + size_t(lb_row(vid)) * kLbRowWords;
    for (uint32_t i = 0; i < kLbSlots; i++) {
        const uint32_t* s = row + i * kLbStride;
        const uint32_t owner = s[0];
        if (owner == 0u) return 0.0f;
        if (owner != vid) continue;
        const uint32_t c = s[6];
        if (c < 2u) return 0.0f;
        const float fc = float(c);
        const float meanL = float(s[7] + s[8] + s[9]) / (3.0f * fc);
        const float meanL2 = float(s[10]) / fc;
        return gmax(meanL2 - meanL * meanL, 0.0f);
    }
    return 0.0f;
}

}  // namespace dev
}  // namespace ve
