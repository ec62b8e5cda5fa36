// emissive.cuh — next-event estimation toward emissive voxels on the device
// (reference src/shd/shade.comp:576-836): the per-scene light registry, the
// single-pick RIS estimator, and ReSTIR DI with per-voxel reservoirs.
//
// Determinism (the reference's versions are order-dependent):
//   * Lights found by a frame's primary hits are staged, sorted by voxel id
//     and appended to the registry at the END of the frame; shading samples
//     the registry as it stood when the frame began (the reference appends
//     during the shade dispatch, in arrival order).
//   * Reservoirs live in a table keyed by the primary voxel id (linear
//     probing, never evicted); during a frame they are only read, and at its
//     end each voxel's reservoir is replaced by the one computed by the
//     voxel's path with the largest path slot (the reference lets every
//     shading invocation store, last writer winning).
#pragma once
#include <cstdint>

#include "ve_device.cuh"

namespace ve {
namespace dev {

// EmissiveVoxel (wavefront.glsl:91-96)
struct EmLight {
    float er, eg, eb;  // mat.color.rgb * mat.emissiveIntensity
    uint32_t vid;      // voxelKey + 1
    uint32_t x, y, z;  // lattice min corner
    uint32_t size;     // lattice extent
};
static_assert(sizeof(EmLight) == 32, "light record");

// One per-voxel reservoir (shade.comp:296-303) with its table key and the
// frame's winning path (largest slot + 1, 0 = none).
struct ResEntry {
    uint32_t key, winner;
    uint32_t light_idx, light_vid, seed;
    float wsum;
    uint32_t m;
    float target;
};
static_assert(sizeof(ResEntry) == 32, "reservoir entry");

struct Reservoir {
    uint32_t light_idx, light_vid, seed;
    float wsum;
    uint32_t m;
    float target;
};

// A path's bounce-0 reservoir, kept until the end-of-frame commit.
struct PathRes {
    uint32_t entry;  // reservoir table entry of the path's primary voxel
    Reservoir r;
    uint32_t scene;
};
static_assert(sizeof(PathRes) == 32, "path reservoir");

constexpr uint32_t kEmCapacity = 4096;  // EMISSIVE_CAPACITY (wavefront.glsl:109)
// Registry claim table: the reference's 8192 rows x 8 probes, here one
// open-addressing table large enough that no claim fails (a failed claim
// would make registration order-dependent).
constexpr uint32_t kEmClaimLog2 = 17;
constexpr uint32_t kEmClaimProbes = 64;
constexpr uint32_t kResLog2 = 20;  // reservoir table entries (2^20 x 32 B)
constexpr uint32_t kResProbes = 64;
constexpr float kMaxContrib = 20.0f;  // firefly clamp of a NEE contribution

__device__ __forceinline__ uint32_t em_hash(uint32_t vid) {  // shade.comp:591
    uint32_t h = vid;
    h ^= h >> 16;
    h *= 0x7feb352du;
    h ^= h >> 15;
    return h;
}

// Claims `vid` in the registry's claim table: true the first time.
__device__ __forceinline__ bool em_claim(uint32_t* claim, uint32_t vid) {
    const uint32_t mask = (1u << kEmClaimLog2) - 1u;
    uint32_t h = em_hash(vid) & mask;
    for (uint32_t q = 0; q < kEmClaimProbes; q++, h = (h + 1u) & mask) {
        const uint32_t prev = atomicCAS(&claim[h], 0u, vid);
        if (prev == 0u) return true;
        if (prev == vid) return false;
    }
    return false;
}

__device__ __forceinline__ float luminance(float r, float g, float b) {
    return (r * 0.2126f + g * 0.7152f) + b * 0.0722f;
}

// rUpdate / rCombine / rCapHistory (shade.comp:316-370)
__device__ __forceinline__ void r_update(Reservoir& r, uint32_t li, uint32_t lv, uint32_t seed, float target, float w,
                                         uint32_t& rng) {
    if (w <= 0.0f) {
        r.m += 1u;
        return;
    }
    r.wsum += w;
    r.m += 1u;
    if (rand01(rng) * r.wsum < w) {
        r.light_idx = li;
        r.light_vid = lv;
        r.seed = seed;
        r.target = target;
    }
}
__device__ __forceinline__ void r_combine(Reservoir& a, const Reservoir& b, float target_at_us, uint32_t& rng) {
    if (b.m == 0u || b.target <= 0.0f || target_at_us <= 0.0f) return;
    const float w = target_at_us * b.wsum / b.target;
    a.wsum += w;
    a.m += b.m;
    if (rand01(rng) * a.wsum < w) {
        a.light_idx = b.light_idx;
        a.light_vid = b.light_vid;
        a.seed = b.seed;
        a.target = target_at_us;
    }
}
__device__ __forceinline__ void r_cap(Reservoir& r, uint32_t max_m) {
    if (r.m > max_m && max_m > 0u) {
        r.wsum = r.wsum * float(max_m) / float(r.m);
        r.m = max_m;
    }
}

// packFaceSeed (shade.comp:376-380): face (4 bits) + u, v (14 bits each)
__device__ __forceinline__ uint32_t pack_face_seed(uint32_t face, float u, float v) {
    const uint32_t ui = uint32_t(gclamp(u, 0.0f, 0.9999f) * 16383.0f);
    const uint32_t vi = uint32_t(gclamp(v, 0.0f, 0.9999f) * 16383.0f);
    return (face & 0xFu) | ((ui & 0x3FFFu) << 4) | ((vi & 0x3FFFu) << 18);
}

// The six faces of a light voxel: outward normal and two tangents
// (shade.comp:397-407, 787-797).
__device__ __forceinline__ void face_frame(uint32_t face, f3& n, f3& t, f3& b) {
    if (face < 2u) {
        n = mk(face == 0u ? 1.0f : -1.0f, 0.0f, 0.0f);
        t = mk(0.0f, 1.0f, 0.0f);
        b = mk(0.0f, 0.0f, 1.0f);
    } else if (face < 4u) {
        n = mk(0.0f, face == 2u ? 1.0f : -1.0f, 0.0f);
        t = mk(1.0f, 0.0f, 0.0f);
        b = mk(0.0f, 0.0f, 1.0f);
    } else {
        n = mk(0.0f, 0.0f, face == 4u ? 1.0f : -1.0f);
        t = mk(1.0f, 0.0f, 0.0f);
        b = mk(0.0f, 1.0f, 0.0f);
    }
}

// A point on the light voxel's surface: face centre + (u - 1/2, v - 1/2) x
// size along the tangents (shade.comp:408-414, 798-804).
__device__ __forceinline__ f3 face_point(const EmLight& L, f3 n, f3 t, f3 b, float u, float v) {
    const float hs = float(L.size) * 0.5f;
    const f3 c = add(mk(float(L.x), float(L.y), float(L.z)), mk(hs, hs, hs));
    const f3 p = add(c, muls(n, hs));
    const f3 q = add(p, muls(t, ((u - 0.5f) * 2.0f) * hs));
    return add(q, muls(b, ((v - 0.5f) * 2.0f) * hs));
}

// unpackLightSamplePoint (shade.comp:392-415)
__device__ __forceinline__ void light_sample_point(uint32_t seed, const EmLight& L, f3& P, f3& N) {
    uint32_t face = seed & 0xFu;
    const float u = float((seed >> 4) & 0x3FFFu) / 16383.0f;
    const float v = float((seed >> 18) & 0x3FFFu) / 16383.0f;
    if (face > 5u) face = 5u;
    f3 t, b;
    face_frame(face, N, t, b);
    P = face_point(L, N, t, b, u, v);
}

// computeTargetPdf (shade.comp:420-435): lum(Le) cos_y area / dist^2, zero
// below the surface's horizon or behind the light's face.
__device__ __forceinline__ float target_pdf(const EmLight& L, uint32_t seed, f3 sp, f3 n) {
    f3 P, N;
    light_sample_point(seed, L, P, N);
    const f3 to = sub(P, sp);
    const float d2 = dot(to, to);
    if (d2 < 1e-6f) return 0.0f;
    const float dist = sqrtf(d2);
    const f3 ld = divs(to, dist);
    const float cx = dot(n, ld);
    if (cx <= 0.0f) return 0.0f;
    const float cy = dot(mk(-ld.x, -ld.y, -ld.z), N);
    if (cy <= 0.0f) return 0.0f;
    const float lum = gmax(luminance(L.er, L.eg, L.eb), 1e-6f);
    const float area = 6.0f * float(L.size * L.size);
    return ((lum * cy) * area) / d2;
}

// neighbourVid (shade.comp:521-531)
__device__ __forceinline__ uint32_t neighbour_vid(uint32_t hx, uint32_t hy, uint32_t hz, uint32_t size, int ox, int oy,
                                                  int oz) {
    const int px = int(hx) + ox * int(size), py = int(hy) + oy * int(size), pz = int(hz) + oz * int(size);
    if (px < 0 || py < 0 || pz < 0) return 0u;
    const uint32_t m = ~(size - 1u);
    const uint32_t sx = uint32_t(px) & m, sy = uint32_t(py) & m, sz = uint32_t(pz) & m;
    const uint32_t p = (sx & 0x3FFu) | ((sy & 0x3FFu) << 10) | ((sz & 0x3FFu) << 20);
    return (hash32(p) & 0x7FFFFFFFu) + 1u;
}

// Reservoir table: probe for `vid` (no insertion).  -1 when absent.
__device__ __forceinline__ int res_find(const ResEntry* t, uint32_t vid) {
    const uint32_t mask = (1u << kResLog2) - 1u;
    uint32_t h = (vid * 0x9E3779B1u) >> (32u - kResLog2);
    for (uint32_t q = 0; q < kResProbes; q++, h = (h + 1u) & mask) {
        const uint32_t k = t[h].key;
        if (k == vid) return int(h);
        if (k == 0u) return -1;
    }
    return -1;
}
// ... with insertion (claim by CAS).  -1 when the probe sequence is full.
__device__ __forceinline__ int res_claim(ResEntry* t, uint32_t vid) {
    const uint32_t mask = (1u << kResLog2) - 1u;
    uint32_t h = (vid * 0x9E3779B1u) >> (32u - kResLog2);
    for (uint32_t q = 0; q < kResProbes; q++, h = (h + 1u) & mask) {
        const uint32_t prev = atomicCAS(&t[h].key, 0u, vid);
        if (prev == 0u || prev == vid) return int(h);
    }
    return -1;
}
// rBufferLoad + lightStillValid (shade.comp:441-515): the committed
// reservoir of `vid` when it exists and its light is still registered.
__device__ __forceinline__ bool res_load(const ResEntry* t, uint32_t vid, const EmLight* lights, uint32_t n_lights,
                                         Reservoir& r) {
    const int e = res_find(t, vid);
    if (e < 0) return false;
    const ResEntry& x = t[e];
    r.light_idx = x.light_idx;
    r.light_vid = x.light_vid;
    r.seed = x.seed;
    r.wsum = x.wsum;
    r.m = x.m;
    r.target = x.target;
    if (r.m == 0u || r.light_idx >= n_lights) return false;
    return lights[r.light_idx].vid == r.light_vid;
}

}  // namespace dev
}  // namespace ve
