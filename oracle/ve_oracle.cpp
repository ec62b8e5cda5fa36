// ve_oracle.cpp — TEST INFRASTRUCTURE ONLY: the CPU oracle for the ray
// pipeline of AnghelusAndrei/VoxelEngine3.0.  It is the checker for the
// product's CUDA kernels and the timed CPU baseline; nothing in the product
// links or calls it.
//
// Every function cites the reference file:line it restates.  The GLSL passes
// cannot execute here (no graphics stack), so this file restates them in
// scalar C++ with a pinned floating-point policy:
//   * compiled with -O2 -ffp-contract=off (no fused multiply-add unless an
//     explicit fmaf is written), IEEE division and sqrt;
//   * GLSL min/max are pinned to glm's expressions: min(a,b) = (b<a)?b:a,
//     max(a,b) = (a<b)?b:a (NaN-propagation is therefore defined);
//   * the Box-Muller RandomDirection (internal.glsl:101-112) uses log/cos,
//     whose last bits differ between libm and CUDA; it is replaced here AND
//     in the kernels by an exact-operation uniform-sphere map whose sin/cos
//     are a project-written Taylor polynomial (Horner form, explicit fmaf)
//     after quadrant reduction.  Deliberate, named deviation.
// Parity pins: the tree build/linearisation and OctreeCPU::raycast are checked
// against the reference's own compiled code (oracle/_ref, see build_ref.sh);
// the GLSL restatements have no reference-side golden vectors.
#include "ve_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <mutex>
#include <stack>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <unordered_set>
#include <vector>

namespace {

// ---------------------------------------------------------------------------
// small float helpers (GLSL semantics pinned as documented above)
// ---------------------------------------------------------------------------
struct f3 {
    float x, y, z;
};
inline f3 mk(float x, float y, float z) { return f3{x, y, z}; }
inline f3 add(f3 a, f3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
inline f3 sub(f3 a, f3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
inline f3 mul(f3 a, f3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
inline f3 muls(f3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
inline f3 divs(f3 a, float s) { return mk(a.x / s, a.y / s, a.z / s); }
inline float gmin(float a, float b) { return (b < a) ? b : a; }
inline float gmax(float a, float b) { return (a < b) ? b : a; }
inline float gclamp(float x, float lo, float hi) { return gmin(gmax(x, lo), hi); }
inline float dot(f3 a, f3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline f3 normalize(f3 v) { return divs(v, std::sqrt(dot(v, v))); }
inline f3 cross(f3 a, f3 b) {
    return mk(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}

// ---------------------------------------------------------------------------
// Node words (src/renderer/octree.hpp:16-37, internal.glsl:1, 18)
// ---------------------------------------------------------------------------
inline bool node_is_node(uint32_t raw) { return raw & 1u; }
inline uint32_t node_next(uint32_t raw) { return (raw & 0xFFFFFFF0u) >> 4; }
inline uint32_t node_material(uint32_t raw) { return (raw & 254u) >> 1; }

struct Scene {
    const uint32_t* words;
    uint64_t n;
    uint32_t depth;
    // ball-normal scenes: the 10-10-10 normal codes their leaves index
    const uint32_t* ncodes = nullptr;
    uint64_t n_ncodes = 0;
    // box that bounce rays are clipped to (scene_clip_box); unbounded by default
    float clip_lo[3] = {-1e30f, -1e30f, -1e30f}, clip_hi[3] = {1e30f, 1e30f, 1e30f};
    // texelFetch on a buffer texture: out-of-range reads return 0.
    uint32_t fetch(uint64_t off) const { return off < n ? words[off] : 0u; }
};

// locate (internal.glsl:30)
inline uint32_t locate(uint32_t x, uint32_t y, uint32_t z, uint32_t p2) {
    return (uint32_t(bool(x & p2)) << 2) | (uint32_t(bool(y & p2)) << 1) | uint32_t(bool(z & p2));
}

// inBounds (internal.glsl:29)
inline bool in_bounds(f3 v, float n) {
    return 0.0f <= v.x && v.x <= n && 0.0f <= v.y && v.y <= n && 0.0f <= v.z && v.z <= n;
}

enum { ST_HIT = 0, ST_ESCAPED = 1, ST_TIMEOUT = 2 };

struct Hit {
    int status;
    uint32_t id, material;
    uint32_t pos[3];
    uint32_t size;
    uint32_t checks;
};

struct RayCounters {
    uint64_t fetch_restart = 0, fetch_min = 0, steps = 0;
};

// Raycast / RaycastCounted (internal.glsl:297-400) with intersect
// (:245-253) and intersect_inside (:255-261).  Returns the termination status
// as well (hit / left the volume / ran out of controlchecks); the reference
// reports only hit-or-not.  `fetch_min` counts a node word only when it
// differs from the word last read at the same descent level (the distinct
// nodes along the ray's monotone DDA walk).
// clip: a bounce ray, for which leaving the volume and running out of
// controlchecks shade alike (shade.comp:558-564), also ends — as having left
// the volume — once its distance passes the exit of the scene's clip box
// along its direction, where it can hit nothing more (scene_clip_box).  This
// changes no result, only the walk the counters see; the device trace does
// the same.
Hit raycast(const Scene& s, f3 o, f3 d, uint32_t controlchecks, RayCounters* rc, bool clip = false) {
    const uint32_t D = s.depth;
    const uint32_t L = 1u << D;
    const float Lf = float(L);
    uint32_t p2c[17];
    for (uint32_t i = 0; i <= D; i++) p2c[i] = L >> i;
    uint32_t last_off[17];
    for (uint32_t i = 0; i <= D; i++) last_off[i] = 0xFFFFFFFFu;

    Hit h{};
    h.status = ST_ESCAPED;
    const f3 inv = mk(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
    o = add(o, muls(d, 4.0f));  // ray.origin += ray.direction * 4  (:361)
    uint32_t q = 0;
    f3 r;
    float t = 0.0f;  // r = d * t + o
    float t_end = 0.0f;
    if (clip) {
        const float tx = ((inv.x > 0.0f ? s.clip_hi[0] : s.clip_lo[0]) - o.x) * inv.x;
        const float ty = ((inv.y > 0.0f ? s.clip_hi[1] : s.clip_lo[1]) - o.y) * inv.y;
        const float tz = ((inv.z > 0.0f ? s.clip_hi[2] : s.clip_lo[2]) - o.z) * inv.z;
        t_end = gmin(gmin(tx, ty), tz);
    }
    if (in_bounds(o, Lf)) {
        r = o;
    } else {
        // intersect(ray, vec3(0), vec3(L))  (:245-253)
        f3 t1 = mul(mk((0.0f - o.x) + 0.001f, (0.0f - o.y) + 0.001f, (0.0f - o.z) + 0.001f), inv);
        f3 t2 = mul(mk((Lf - o.x) - 0.001f, (Lf - o.y) - 0.001f, (Lf - o.z) - 0.001f), inv);
        f3 tmn = mk(gmin(t1.x, t2.x), gmin(t1.y, t2.y), gmin(t1.z, t2.z));
        f3 tmx = mk(gmax(t1.x, t2.x), gmax(t1.y, t2.y), gmax(t1.z, t2.z));
        float t_enter = gmax(gmax(tmn.x, tmn.y), tmn.z);
        float t_exit = gmin(gmin(tmx.x, tmx.y), tmx.z);
        q++;
        if (t_exit < t_enter || t_exit < 0.0f) {
            h.checks = q;
            return h;
        }
        r = add(muls(d, t_enter), o);
        t = t_enter;
    }
    bool clipped = false;
    while (in_bounds(r, Lf) && !(clipped = clip && t > t_end) && q++ <= controlchecks) {
        if (rc) rc->steps++;
        const uint32_t ux = uint32_t(r.x), uy = uint32_t(r.y), uz = uint32_t(r.z);
        uint32_t off = 0, depth = 0, size = 0;
        bool found = false;
        for (; depth < D; depth++) {
            off += locate(ux, uy, uz, p2c[depth]);
            const uint32_t raw = s.fetch(off);
            if (rc) {
                rc->fetch_restart++;
                if (last_off[depth] != off) { rc->fetch_min++; last_off[depth] = off; }
            }
            if (!node_is_node(raw)) {
                size = p2c[depth];
                found = true;
                break;
            }
            off = node_next(raw);
        }
        uint32_t px, py, pz;
        if (!found) {
            off += locate(ux, uy, uz, p2c[depth]);
            const uint32_t raw = s.fetch(off);
            if (rc) {
                rc->fetch_restart++;
                if (last_off[depth] != off) { rc->fetch_min++; last_off[depth] = off; }
            }
            size = p2c[depth];
            px = ux & ~(size - 1u); py = uy & ~(size - 1u); pz = uz & ~(size - 1u);
            if (node_material(raw) != 0u) {
                h.status = ST_HIT;
                h.id = off;
                h.material = node_material(raw);
                h.pos[0] = px; h.pos[1] = py; h.pos[2] = pz;
                h.size = size;
                h.checks = q;
                return h;
            }
        } else {
            px = ux & ~(size - 1u); py = uy & ~(size - 1u); pz = uz & ~(size - 1u);
        }
        // intersect_inside(ray, pos, pos + size)  (:255-261)
        const f3 bmin = mk(float(px), float(py), float(pz));
        const float fs = float(size);
        const f3 bmax = mk(bmin.x + fs, bmin.y + fs, bmin.z + fs);
        f3 t1 = mul(mk((bmin.x - o.x) - 0.001f, (bmin.y - o.y) - 0.001f, (bmin.z - o.z) - 0.001f), inv);
        f3 t2 = mul(mk((bmax.x - o.x) + 0.001f, (bmax.y - o.y) + 0.001f, (bmax.z - o.z) + 0.001f), inv);
        f3 tmx = mk(gmax(t1.x, t2.x), gmax(t1.y, t2.y), gmax(t1.z, t2.z));
        float t_exit = gmin(gmin(tmx.x, tmx.y), tmx.z);
        r = add(muls(d, t_exit), o);
        t = t_exit;
    }
    h.status = (in_bounds(r, Lf) && !clipped) ? ST_TIMEOUT : ST_ESCAPED;
    h.checks = q;
    return h;
}

// The box bounce rays are clipped to (a bound of this build, not of the
// reference).  Levels 0..T0-1 (T0 = min(10, D), none below depth 3) are
// the device's top-table levels; a level-(T0-1) cell whose words at those
// levels are all internal can end a descent on a material voxel, no other
// in-range cell can (words above level D are never tested for a material).
// The box of those cells, widened by one voxel, unless a position with a
// coordinate equal to 2^D (which the bounds test admits; its level-0 read
// goes to root words 1..7) ends on a material voxel: then, as for depths
// above 12 where the faces are not searched, no box applies.
void scene_clip_box(Scene& s) {
    const uint32_t D = s.depth;
    const uint32_t T0 = D < 3u ? 0u : std::min(10u, D);
    if (T0 == 0 || D > 12) return;
    const uint32_t L = 1u << D, sh = D - T0 + 1u;
    uint32_t lo[3] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu}, hi[3] = {0u, 0u, 0u};
    struct C { uint32_t off, k, x, y, z; };
    std::vector<C> st{{0u, 0u, 0u, 0u, 0u}};
    while (!st.empty()) {
        const C c = st.back();
        st.pop_back();
        const uint32_t raw = s.fetch(c.off);
        if (!(raw & 1u)) continue;
        if (c.k == T0 - 1u) {
            const uint32_t v[3] = {c.x >> sh, c.y >> sh, c.z >> sh};
            for (int a = 0; a < 3; a++) {
                lo[a] = std::min(lo[a], v[a]);
                hi[a] = std::max(hi[a], v[a]);
            }
            continue;
        }
        const uint32_t next = node_next(raw), half = L >> (c.k + 1u);
        for (uint32_t i = 0; i < 8; i++)
            st.push_back({next + i, c.k + 1u, c.x + ((i & 4) ? half : 0u), c.y + ((i & 2) ? half : 0u),
                          c.z + ((i & 1) ? half : 0u)});
    }
    // the faces {x, y or z = 2^D}: the descent of raycast at each integer position
    for (uint32_t f = 0; f < 3; f++)
        for (uint32_t u = 0; u <= L; u++)
            for (uint32_t v = 0; v <= L; v++) {
                const uint32_t x = f == 0 ? L : u, y = f == 1 ? L : (f == 0 ? u : v), z = f == 2 ? L : v;
                uint32_t off = 0;
                bool internal = true;
                for (uint32_t k = 0; k < D && internal; k++) {
                    const uint32_t raw = s.fetch(off + locate(x, y, z, L >> k));
                    internal = node_is_node(raw);
                    off = node_next(raw);
                }
                if (internal && node_material(s.fetch(off + locate(x, y, z, 1u))) != 0u) return;
            }
    for (int a = 0; a < 3; a++) {
        if (lo[0] > hi[0]) {  // no cell can be hit: any box is exact
            s.clip_lo[a] = -1.0f;
            s.clip_hi[a] = 1.0f;
        } else {
            s.clip_lo[a] = float(lo[a] << sh) - 1.0f;
            s.clip_hi[a] = float((hi[a] + 1u) << sh) + 1.0f;
        }
    }
}

// hash + voxelKey (internal.glsl:263-291)
inline uint32_t hash32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
inline uint32_t voxel_key(const uint32_t pos[3]) {
    uint32_t p = pos[0] | (pos[1] << 10) | (pos[2] << 20);
    return hash32(p) & 0x7FFFFFFFu;
}

// halton + rand (internal.glsl:57-89)
const uint32_t kHaltonBases[16] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53};
inline float halton(uint32_t i, uint32_t b) {
    float f = 1.0f, r = 0.0f;
    for (int k = 0; k < 24 && i > 0u; k++) {
        f /= float(b);
        uint32_t q = i / b;
        r += f * float(i - q * b);
        i = q;
    }
    return r;
}
inline float rand01(uint32_t& state) {
    uint32_t dim = state & 0xFFu;
    uint32_t sample_idx = state >> 8;
    state = (sample_idx << 8) | ((dim + 1u) & 0xFFu);
    uint32_t base = kHaltonBases[dim & 15u];
    uint32_t effective = sample_idx ^ ((dim >> 4) * 0x9E3779B9u);
    return halton(effective, base);
}

// Project-written sin/cos of 2*pi*u for u in [0,1]: quadrant reduction
// (exact: x = 4u, q = floor(x), f = x - q) then Taylor polynomials of
// sin/cos on [0, pi/2) in Horner form with explicit fmaf (degree 11 / 12;
// truncation error < 6e-8).  Replaces the reference's cos/log sampling.
inline void sincos_turn(float u, float* s_out, float* c_out) {
    const float x = u * 4.0f;
    const float qf = std::floor(x);
    const int q = int(qf) & 3;
    const float t = (x - qf) * 0x1.921fb6p+0f;
    const float t2 = t * t;
    float ps = std::fmaf(t2, -0x1.ae6456p-26f, 0x1.71de3ap-19f);
    ps = std::fmaf(t2, ps, -0x1.a01a02p-13f);
    ps = std::fmaf(t2, ps, 0x1.111112p-7f);
    ps = std::fmaf(t2, ps, -0x1.555556p-3f);
    const float s = std::fmaf(t * t2, ps, t);
    float pc = std::fmaf(t2, 0x1.1eed8ep-29f, -0x1.27e4fcp-22f);
    pc = std::fmaf(t2, pc, 0x1.a01a02p-16f);
    pc = std::fmaf(t2, pc, -0x1.6c16c2p-10f);
    pc = std::fmaf(t2, pc, 0x1.555556p-5f);
    pc = std::fmaf(t2, pc, -0x1p-1f);
    const float c = std::fmaf(t2, pc, 1.0f);
    switch (q) {
        case 0: *s_out = s; *c_out = c; break;
        case 1: *s_out = c; *c_out = -s; break;
        case 2: *s_out = -s; *c_out = -c; break;
        default: *s_out = -c; *c_out = s; break;
    }
}

// Uniform direction on the unit sphere from two rand() draws; stands in for
// RandomDirection (internal.glsl:107-112).
inline f3 uniform_sphere(uint32_t& rng) {
    const float u1 = rand01(rng);
    const float u2 = rand01(rng);
    const float z = 1.0f - 2.0f * u1;
    const float rr = std::sqrt(gmax(1.0f - z * z, 0.0f));
    float sn, cs;
    sincos_turn(u2, &sn, &cs);
    return mk(rr * cs, rr * sn, z);
}

// normalize(N + RandomDirection) (shade.comp:869) with a zero-length guard.
inline f3 cosine_direction(f3 n, uint32_t& rng) {
    const f3 v = add(n, uniform_sphere(rng));
    const float d2 = dot(v, v);
    if (!(d2 > 1e-12f)) return n;
    return divs(v, std::sqrt(d2));
}

// Material (src/renderer/material.hpp:17-25; std140 64-B stride)
struct Material {
    float color[4];
    float specular_color[4];
    float roughness, specular, metallic;
    int32_t emissive;
    float emissive_intensity;
    float pad[3];
};
static_assert(sizeof(Material) == 64, "material stride");

// x^e for x in (0, 1], e > 0: exp2(e log2 x) with the atanh series of the
// mantissa's logarithm and the Taylor series of 2^f (explicit fma), the same
// operation sequence as the device's pow_unit; results below 2^-125 are 0.
inline float pow_unit(float x, float e) {
    if (x != x) return x;  // NaN stays NaN
    uint32_t bits;
    std::memcpy(&bits, &x, 4);
    int ex = int(bits >> 23) - 127;
    const uint32_t mb = (bits & 0x007FFFFFu) | 0x3F800000u;
    float m;
    std::memcpy(&m, &mb, 4);
    if (m > 1.41421356f) {
        m = m * 0.5f;
        ex += 1;
    }
    const float s = (m - 1.0f) / (m + 1.0f);
    const float s2 = s * s;
    float p = std::fmaf(s2, 0.0769230769f, 0.0909090909f);
    p = std::fmaf(s2, p, 0.111111111f);
    p = std::fmaf(s2, p, 0.142857143f);
    p = std::fmaf(s2, p, 0.2f);
    p = std::fmaf(s2, p, 0.333333333f);
    const float lnm = 2.0f * std::fmaf(s * s2, p, s);
    const float y = e * (float(ex) + lnm * 1.44269504f);
    if (!(y > -125.0f)) return 0.0f;
    const float n = std::floor(y + 0.5f);
    const float t = (y - n) * 0.693147181f;
    float q = std::fmaf(t, 2.48015873e-5f, 1.98412698e-4f);
    q = std::fmaf(t, q, 1.38888889e-3f);
    q = std::fmaf(t, q, 8.33333333e-3f);
    q = std::fmaf(t, q, 4.16666667e-2f);
    q = std::fmaf(t, q, 0.166666667f);
    q = std::fmaf(t, q, 0.5f);
    q = std::fmaf(t, q, 1.0f);
    q = std::fmaf(t, q, 1.0f);
    uint32_t qb;
    std::memcpy(&qb, &q, 4);
    qb += uint32_t(int(n)) << 23;
    float r;
    std::memcpy(&r, &qb, 4);
    return r;
}

// EvaluateBRDF (internal.glsl:120-149)
inline f3 evaluate_brdf(f3 V, f3 L, f3 N, f3 albedo, float roughness, float metallic,
                        float specular_intensity) {
    const float NdotL = gmax(dot(N, L), 0.001f);
    if (NdotL < 0.001f) return mk(0, 0, 0);
    const float rc = gmax(roughness, 0.01f);
    const float spec_exp = 2.0f / (rc * rc);
    const f3 H = normalize(sub(L, V));
    const float NdotH = gmax(dot(N, H), 0.001f);
    const float spec_norm = (spec_exp + 2.0f) * 0.15915494f;
    const float specular = spec_norm * pow_unit(NdotH, spec_exp);
    const float kS = specular_intensity * metallic;
    const float kD = 1.0f - kS * 0.5f;
    const f3 diffuse = muls(muls(albedo, kD), 0.31831f);
    const float sp = specular * kS;
    return muls(mk(diffuse.x + sp, diffuse.y + sp, diffuse.z + sp), NdotL);
}

// smithG1GGX / sampleGGXVNDF / ggxThroughput (internal.glsl:165-239);
// pow(x, 5.0) is evaluated as x*x*x*x*x, sin/cos via sincos_turn.
inline float smith_g1(float NdotX, float a) {
    const float a2 = a * a;
    return 2.0f * NdotX / (NdotX + std::sqrt(a2 + (1.0f - a2) * NdotX * NdotX));
}
inline f3 sample_ggx_vndf(f3 N, f3 V, float roughness, uint32_t& rng) {
    const float a = gmax(roughness * roughness, 0.001f);
    const f3 up = std::fabs(N.z) < 0.999f ? mk(0, 0, 1) : mk(1, 0, 0);
    const f3 T = normalize(cross(up, N));
    const f3 B = cross(N, T);
    const f3 Vl = mk(dot(V, T), dot(V, B), dot(V, N));
    const f3 Vh = normalize(mk(a * Vl.x, a * Vl.y, Vl.z));
    const float lensq = Vh.x * Vh.x + Vh.y * Vh.y;
    f3 T1;
    if (lensq > 0.0f) {
        const float is = 1.0f / std::sqrt(lensq);
        T1 = mk(-Vh.y * is, Vh.x * is, 0.0f);
    } else {
        T1 = mk(1, 0, 0);
    }
    const f3 T2 = cross(Vh, T1);
    const float r1 = rand01(rng);
    const float r2 = rand01(rng);
    const float r = std::sqrt(r1);
    float sn, cs;
    sincos_turn(r2, &sn, &cs);
    const float t1 = r * cs;
    float t2 = r * sn;
    const float s = 0.5f * (1.0f + Vh.z);
    t2 = (1.0f - s) * std::sqrt(gmax(1.0f - t1 * t1, 0.0f)) + s * t2;
    const float w = std::sqrt(gmax(0.0f, 1.0f - t1 * t1 - t2 * t2));
    const f3 Nh = add(add(muls(T1, t1), muls(T2, t2)), muls(Vh, w));
    const f3 Hl = normalize(mk(a * Nh.x, a * Nh.y, gmax(0.0f, Nh.z)));
    return add(add(muls(T, Hl.x), muls(B, Hl.y)), muls(N, Hl.z));
}
inline f3 ggx_throughput(f3 N, f3 V, f3 L, f3 H, float roughness, f3 F0) {
    const float NdotL = gmax(dot(N, L), 0.001f);
    const float VdotH = gmax(dot(V, H), 0.001f);
    const float a = roughness * roughness;
    const float x = 1.0f - VdotH;
    const float x2 = x * x;
    const float x5 = x2 * x2 * x;
    const f3 F = mk(F0.x + (1.0f - F0.x) * x5, F0.y + (1.0f - F0.y) * x5, F0.z + (1.0f - F0.z) * x5);
    return muls(F, smith_g1(NdotL, a));
}
// reflect(I, N) = I - 2*dot(N,I)*N (GLSL spec)
inline f3 reflect(f3 I, f3 N) { return sub(I, muls(N, 2.0f * dot(N, I))); }

// ---------------------------------------------------------------------------
// Normals.  The reference computes per-voxel normals in normal.comp
// (:55-95) as normalize(sum of offsets of EMPTY neighbours) with an L2-ball
// neighbourhood and caches them 10-10-10 packed; the benchmark method uses the
// full 3x3x3 neighbourhood and keeps the integer sum in the leaf word's unused
// 24-bit `normal` field (octree.hpp:29): bits 8-12 x, 13-17 y, 18-22 z (5-bit
// two's complement, each in [-9, 9]), bit 31 = "normal present".
// ---------------------------------------------------------------------------
// lookupOccupied (normal.comp:55-70)
bool lookup_occupied(const Scene& s, int64_t x, int64_t y, int64_t z) {
    const uint32_t L = 1u << s.depth;
    if (x < 0 || y < 0 || z < 0 || x >= L || y >= L || z >= L) return false;
    uint32_t off = 0, raw;
    for (uint32_t d = 0; d < s.depth; d++) {
        off += locate(uint32_t(x), uint32_t(y), uint32_t(z), L >> d);
        raw = s.fetch(off);
        if (!(raw & 1u)) return bool((raw >> 1) & 0x7Fu);
        off = (raw >> 4) & 0x0FFFFFFFu;
    }
    off += locate(uint32_t(x), uint32_t(y), uint32_t(z), L >> s.depth);
    raw = s.fetch(off);
    return bool((raw >> 1) & 0x7Fu);
}

uint32_t encode_normal_field(int ix, int iy, int iz) {
    return ((uint32_t(ix) & 31u) << 8) | ((uint32_t(iy) & 31u) << 13) | ((uint32_t(iz) & 31u) << 18) |
           (1u << 31);
}
inline int sext5(uint32_t v) { return (v & 16u) ? int(v) - 32 : int(v); }

// Shading normal for a hit: decode the gradient sum, then normalize ->
// packNormalAccum (normal.comp:90-95) -> UnpackNormal (internal.glsl:22-28)
// -> normalize, as shade.comp:267 reads it.  Leaves without a stored normal
// use the face-normal fallback of lookupNormal (shade.comp:271-274).
// UnpackNormal (internal.glsl:22-28) of a 10-10-10 code, then normalize.
f3 unpack_normal(uint32_t p) {
    const f3 u = mk(float((p >> 22) & 0x3FFu) / 511.0f - 1.0f, float((p >> 12) & 0x3FFu) / 511.0f - 1.0f,
                    float((p >> 2) & 0x3FFu) / 511.0f - 1.0f);
    return normalize(u);
}

// index + 1 of a ball-normal leaf's code in the scene's table (0: none)
inline uint32_t ball_index(uint32_t leaf_word) { return (leaf_word >> 31) ? 0u : (leaf_word >> 8) & 0x7FFFFFu; }

// whether the leaf word carries a stored normal (either mode)
inline bool has_normal(uint32_t leaf_word) { return (leaf_word >> 31) || ball_index(leaf_word) != 0u; }

f3 shading_normal(const Scene& s, uint32_t leaf_word, f3 ray_dir) {
    const uint32_t bi = ball_index(leaf_word);
    if (bi != 0u && bi - 1u < s.n_ncodes) return unpack_normal(s.ncodes[bi - 1u]);
    if (!(leaf_word >> 31)) {
        const f3 a = mk(std::fabs(ray_dir.x), std::fabs(ray_dir.y), std::fabs(ray_dir.z));
        auto sgn = [](float v) { return v > 0.0f ? 1.0f : (v < 0.0f ? -1.0f : 0.0f); };
        if (a.x > a.y && a.x > a.z) return mk(-sgn(ray_dir.x), 0.0f, 0.0f);
        if (a.y > a.z) return mk(0.0f, -sgn(ray_dir.y), 0.0f);
        return mk(0.0f, 0.0f, -sgn(ray_dir.z));
    }
    const f3 acc = mk(float(sext5((leaf_word >> 8) & 31u)), float(sext5((leaf_word >> 13) & 31u)),
                      float(sext5((leaf_word >> 18) & 31u)));
    const float len = std::sqrt(dot(acc, acc));
    const f3 n = len > 0.001f ? divs(acc, len) : mk(0.0f, 1.0f, 0.0f);
    auto pack = [](float c) {
        int v = int(std::round((c + 1.0f) * 511.0f));
        v = v < 0 ? 0 : (v > 1022 ? 1022 : v);
        return uint32_t(v);
    };
    const uint32_t px = pack(n.x), py = pack(n.y), pz = pack(n.z);
    const f3 u = mk(float(px) / 511.0f - 1.0f, float(py) / 511.0f - 1.0f, float(pz) / 511.0f - 1.0f);
    return normalize(u);
}

// ---------------------------------------------------------------------------
// Pointer octree restated from src/octree_cpu.cpp (insert/insertR :33-64,
// remove/removeR :66-98, lookup :100-112) and src/renderer/octree.cpp
// (set :127-166, linearizeNode :170-217).
// ---------------------------------------------------------------------------
struct PNode {
    PNode* child[8] = {};
    uint8_t count = 0;
    uint32_t material = 0;
};
struct PTree {
    PNode* root = nullptr;
    uint32_t depth;
    uint32_t p2r[18];
    std::vector<std::unique_ptr<PNode>> pool;
    explicit PTree(uint32_t d) : depth(d) {
        uint32_t p = 1;
        for (int i = int(d); i >= 1; i--) { p2r[i] = p; p <<= 1; }
        p2r[0] = p;
    }
    PNode* alloc() { pool.emplace_back(new PNode()); return pool.back().get(); }
    void insert(uint32_t x, uint32_t y, uint32_t z, uint32_t m) {
        const uint32_t b = 1u << depth;
        if (x >= b || y >= b || z >= b) return;
        if (!root) root = alloc();
        PNode* n = root;
        for (uint32_t level = 1; level <= depth; level++) {
            const uint32_t idx = locate(x, y, z, p2r[level]);
            if (!n->child[idx]) { n->child[idx] = alloc(); n->count++; }
            n = n->child[idx];
        }
        n->material = m;
        n->count = 0;
    }
    // Octree::set slot order: slot 0 root, 1-8 root children (processed in
    // order 0..7), each internal node gets an 8-slot block at `size` in
    // iterative-DFS LIFO order (children pushed 0..7, popped 7..0).
    std::vector<uint32_t> linearize(uint32_t* size_out, uint32_t* nvox) const {
        std::vector<uint32_t> data(9, 0u);
        uint32_t size = 9, nv = 0;
        if (!root) { *size_out = 9; *nvox = 0; return data; }
        data[0] = 1u | ((uint32_t(root->count) & 7u) << 1) | (1u << 4);
        for (int i = 0; i < 8; i++) {
            std::stack<std::tuple<PNode*, uint32_t, uint32_t>> st;
            st.push({root->child[i], uint32_t(i + 1), 2u});
            while (!st.empty()) {
                auto [cn, off, lv] = st.top();
                st.pop();
                if (!cn) continue;
                if (lv > depth || (cn->material != 0 && cn->count == 0)) {
                    if (cn->material == 0) continue;
                    if (data.size() <= off) data.resize(off + 1, 0u);
                    data[off] = ((cn->material & 0x7Fu) << 1);
                    nv++;
                } else {
                    const uint32_t block = size;
                    size += 8;
                    if (data.size() < size) data.resize(size, 0u);
                    data[off] = 1u | ((uint32_t(cn->count) & 7u) << 1) | (block << 4);
                    for (int k = 0; k < 8; k++) st.push({cn->child[k], block + uint32_t(k), lv + 1});
                }
            }
        }
        data.resize(size, 0u);
        *size_out = size;
        *nvox = nv;
        return data;
    }
};

// ---------------------------------------------------------------------------
// FP64 radiance cache: the re-accumulation reference for the product's FP32
// hash cache.  Keyed by voxel id (voxelKey + 1).
// ---------------------------------------------------------------------------
struct CacheEntry {
    uint64_t count = 0;
    double weight = 0, r = 0, g = 0, b = 0, l2 = 0;
};
// Sharded by vid so the merge and the decay run in parallel; within a
// shard, deposits merge in (thread, row) order: deterministic.
constexpr uint32_t kShards = 64;
inline uint32_t shard_of(uint32_t vid) { return hash32(vid) & (kShards - 1); }
struct Cache {
    std::unordered_map<uint32_t, CacheEntry> map[kShards];
    const CacheEntry* find(uint32_t vid) const {
        const auto& m = map[shard_of(vid)];
        auto it = m.find(vid);
        return it == m.end() ? nullptr : &it->second;
    }
    size_t size() const {
        size_t n = 0;
        for (const auto& m : map) n += m.size();
        return n;
    }
};

template <typename F>
void run_parallel(uint32_t n, uint32_t threads, F&& fn) {
    if (threads <= 1) {
        for (uint32_t i = 0; i < n; i++) fn(i);
        return;
    }
    std::vector<std::thread> th;
    for (uint32_t t = 0; t < threads; t++)
        th.emplace_back([&, t] {
            for (uint32_t i = t; i < n; i += threads) fn(i);
        });
    for (auto& x : th) x.join();
}

struct Deposit {
    uint32_t vid;
    float rgb[3];
    uint32_t slot;      // the path's slot (lBuffer frames apply deposits in slot order)
    float d[3], e[3];   // clamped direct and indirect radiance (lBuffer frames)
};

struct PathOut {
    f3 direct{0, 0, 0}, indirect{0, 0, 0};
};

// ---------------------------------------------------------------------------
// Emissive NEE (shade.comp:576-836): the light registry, the single-pick RIS
// estimator and ReSTIR DI with per-voxel reservoirs, under the product's
// deterministic rules: lights seen by a frame's primary hits join the
// registry at the end of the frame (sorted by vid, up to 4096), reservoirs
// are read as committed by earlier frames and each voxel keeps the reservoir
// of its frame's largest path slot.
// ---------------------------------------------------------------------------
constexpr uint32_t kEmCapacity = 4096;  // EMISSIVE_CAPACITY (wavefront.glsl:109)
constexpr uint32_t kFrameEmissive = 128;  // VE_FRAME_EMISSIVE
constexpr uint32_t kRestirEnable = 1, kRestirTemporal = 2, kRestirSpatial = 4;

struct EmLight {  // EmissiveVoxel (wavefront.glsl:91-96)
    float e[3];
    uint32_t vid;
    uint32_t pos[3];
    uint32_t size;
};
struct Reservoir {  // shade.comp:296-303
    uint32_t light_idx = 0, light_vid = 0, seed = 0;
    float wsum = 0.0f;
    uint32_t m = 0;
    float target = 0.0f;
};
struct ResRecord {
    uint32_t vid, slot;
    Reservoir r;
};
// A frame's emissive-NEE inputs (the registry and reservoirs as the frame
// began) and one thread's outputs.
struct EmFrame {
    const std::vector<EmLight>* lights = nullptr;
    const std::unordered_map<uint32_t, Reservoir>* res = nullptr;
    std::vector<EmLight> staged;
    std::vector<ResRecord> records;
    uint64_t nee = 0;
};

inline float luminance(const float e[3]) { return (e[0] * 0.2126f + e[1] * 0.7152f) + e[2] * 0.0722f; }

// rUpdate / rCombine / rCapHistory (shade.comp:316-370)
inline void r_update(Reservoir& r, uint32_t li, uint32_t lv, uint32_t seed, float target, float w, uint32_t& rng) {
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
inline void r_combine(Reservoir& a, const Reservoir& b, float target_at_us, uint32_t& rng) {
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
inline void r_cap(Reservoir& r, uint32_t max_m) {
    if (r.m > max_m && max_m > 0u) {
        r.wsum = r.wsum * float(max_m) / float(r.m);
        r.m = max_m;
    }
}
// packFaceSeed (shade.comp:376-380)
inline uint32_t pack_face_seed(uint32_t face, float u, float v) {
    const uint32_t ui = uint32_t(gclamp(u, 0.0f, 0.9999f) * 16383.0f);
    const uint32_t vi = uint32_t(gclamp(v, 0.0f, 0.9999f) * 16383.0f);
    return (face & 0xFu) | ((ui & 0x3FFFu) << 4) | ((vi & 0x3FFFu) << 18);
}
// face normal and tangents (shade.comp:397-407)
inline void face_frame(uint32_t face, f3& n, f3& t, f3& b) {
    if (face < 2u) {
        n = mk(face == 0u ? 1.0f : -1.0f, 0, 0); t = mk(0, 1, 0); b = mk(0, 0, 1);
    } else if (face < 4u) {
        n = mk(0, face == 2u ? 1.0f : -1.0f, 0); t = mk(1, 0, 0); b = mk(0, 0, 1);
    } else {
        n = mk(0, 0, face == 4u ? 1.0f : -1.0f); t = mk(1, 0, 0); b = mk(0, 1, 0);
    }
}
// fCenter + fNormal*halfSize + (u-0.5)*2*halfSize*fT + (v-0.5)*2*halfSize*fB
// (shade.comp:408-414, 798-804)
inline f3 face_point(const EmLight& L, f3 n, f3 t, f3 b, float u, float v) {
    const float hs = float(L.size) * 0.5f;
    const f3 c = add(mk(float(L.pos[0]), float(L.pos[1]), float(L.pos[2])), mk(hs, hs, hs));
    const f3 p = add(c, muls(n, hs));
    const f3 q = add(p, muls(t, ((u - 0.5f) * 2.0f) * hs));
    return add(q, muls(b, ((v - 0.5f) * 2.0f) * hs));
}
// unpackLightSamplePoint (shade.comp:392-415)
inline void light_sample_point(uint32_t seed, const EmLight& L, f3& P, f3& N) {
    uint32_t face = seed & 0xFu;
    const float u = float((seed >> 4) & 0x3FFFu) / 16383.0f;
    const float v = float((seed >> 18) & 0x3FFFu) / 16383.0f;
    if (face > 5u) face = 5u;
    f3 t, b;
    face_frame(face, N, t, b);
    P = face_point(L, N, t, b, u, v);
}
// computeTargetPdf (shade.comp:420-435)
inline float target_pdf(const EmLight& L, uint32_t seed, f3 sp, f3 n) {
    f3 P, N;
    light_sample_point(seed, L, P, N);
    const f3 to = sub(P, sp);
    const float d2 = dot(to, to);
    if (d2 < 1e-6f) return 0.0f;
    const float dist = std::sqrt(d2);
    const f3 ld = divs(to, dist);
    const float cx = dot(n, ld);
    if (cx <= 0.0f) return 0.0f;
    const float cy = dot(mk(-ld.x, -ld.y, -ld.z), N);
    if (cy <= 0.0f) return 0.0f;
    const float lum = gmax(luminance(L.e), 1e-6f);
    const float area = 6.0f * float(L.size * L.size);
    return ((lum * cy) * area) / d2;
}
// neighbourVid (shade.comp:521-531)
inline uint32_t neighbour_vid(const uint32_t pos[3], uint32_t size, int ox, int oy, int oz) {
    const int px = int(pos[0]) + ox * int(size), py = int(pos[1]) + oy * int(size), pz = int(pos[2]) + oz * int(size);
    if (px < 0 || py < 0 || pz < 0) return 0u;
    const uint32_t m = ~(size - 1u);
    const uint32_t sx = uint32_t(px) & m, sy = uint32_t(py) & m, sz = uint32_t(pz) & m;
    const uint32_t p = (sx & 0x3FFu) | ((sy & 0x3FFu) << 10) | ((sz & 0x3FFu) << 20);
    return (hash32(p) & 0x7FFFFFFFu) + 1u;
}
// rBufferLoad + lightStillValid (shade.comp:441-515)
inline bool res_load(const EmFrame& em, uint32_t vid, Reservoir& r) {
    auto it = em.res->find(vid);
    if (it == em.res->end()) return false;
    r = it->second;
    const uint32_t n = uint32_t(std::min<size_t>(em.lights->size(), kEmCapacity));
    if (r.m == 0u || r.light_idx >= n) return false;
    return (*em.lights)[r.light_idx].vid == r.light_vid;
}
inline f3 clamp_contrib(f3 c) { return mk(gmin(c.x, 20.0f), gmin(c.y, 20.0f), gmin(c.z, 20.0f)); }

// NEE toward the registered lights at a non-emissive hit of bounce b < 2;
// the shadow ray must hit the light's voxel (RaycastVisibilityToVoxel,
// internal.glsl:406-410).  Adds to direct (b == 0) or indirect radiance.
void emissive_nee(const Scene& s, const ov_frame_params& P, EmFrame& em, uint32_t slot, uint32_t primary_vid,
                  uint32_t b, const Hit& hit, f3 N, f3 sp, f3 dir, f3 tp, f3 albedo, const Material& m,
                  uint32_t& rng, f3& direct, f3& indirect, ov_stats* st, RayCounters* rc) {
    const std::vector<EmLight>& lights = *em.lights;
    const uint32_t n_lights = uint32_t(std::min<size_t>(lights.size(), kEmCapacity));
    if (n_lights == 0u) return;
    bool have = false;
    f3 contrib{0, 0, 0}, ld{0, 0, 0};
    uint32_t target_vid = 0;
    if ((P.restir & kRestirEnable) && b == 0u) {
        Reservoir res;
        const uint32_t n_m = std::max(P.restir_m, 1u);
        const float inv_src = float(n_lights) * 6.0f;
        for (uint32_t k = 0; k < n_m; k++) {
            uint32_t pick = uint32_t(rand01(rng) * float(n_lights));
            if (pick >= n_lights) pick = n_lights - 1u;
            const EmLight& cand = lights[pick];
            uint32_t face = uint32_t(rand01(rng) * 6.0f);
            if (face >= 6u) face = 5u;
            const float uu = rand01(rng);
            const float vv = rand01(rng);
            const uint32_t seed = pack_face_seed(face, uu, vv);
            const float target = target_pdf(cand, seed, sp, N);
            r_update(res, pick, cand.vid, seed, target, target * inv_src, rng);
        }
        if (P.restir & kRestirTemporal) {
            Reservoir t;
            if (res_load(em, primary_vid, t)) {
                r_cap(t, P.restir_max_m);
                r_combine(res, t, t.target, rng);
            }
        }
        if ((P.restir & kRestirSpatial) && P.restir_spatial_neighbors > 0u) {
            const f3 up = std::fabs(N.z) < 0.999f ? mk(0, 0, 1) : mk(1, 0, 0);
            const f3 T = normalize(cross(up, N));
            const f3 B = cross(N, T);
            const uint32_t K = std::min(P.restir_spatial_neighbors, 6u);
            for (uint32_t k = 0; k < K; k++) {
                const float ua = rand01(rng);
                const float rr = P.restir_spatial_radius * std::sqrt(rand01(rng));
                float sn, cs;
                sincos_turn(ua, &sn, &cs);
                const f3 off = muls(add(muls(T, cs), muls(B, sn)), rr);
                const int ox = int(std::round(off.x)), oy = int(std::round(off.y)), oz = int(std::round(off.z));
                if (ox == 0 && oy == 0 && oz == 0) continue;
                const uint32_t nvid = neighbour_vid(hit.pos, 1u, ox, oy, oz);
                if (nvid == 0u || nvid == primary_vid) continue;
                Reservoir nb;
                if (!res_load(em, nvid, nb)) continue;
                const float tu = target_pdf(lights[nb.light_idx], nb.seed, sp, N);
                if (tu <= 0.0f) continue;
                r_cap(nb, P.restir_max_m);
                r_combine(res, nb, tu, rng);
            }
        }
        if (res.m > 0u && res.target > 0.0f) {
            const EmLight& L = lights[res.light_idx];
            if (L.vid == res.light_vid) {
                f3 LP, LN;
                light_sample_point(res.seed, L, LP, LN);
                const f3 to = sub(LP, sp);
                const float d2 = dot(to, to);
                const float dist = std::sqrt(gmax(d2, 1e-12f));
                if (dist > 1e-3f) {
                    const f3 l = divs(to, dist);
                    const float cx = gmax(dot(N, l), 0.0f);
                    const float cy = gmax(dot(mk(-l.x, -l.y, -l.z), LN), 0.0f);
                    if (cx > 0.0f && cy > 0.0f) {
                        const f3 brdf = evaluate_brdf(dir, l, N, albedo, m.roughness, m.metallic, m.specular);
                        const float W = res.wsum / (float(res.m) * res.target);
                        const float sz2 = float(L.size * L.size);
                        const float geom = cy / gmax(d2, 1e-6f);
                        contrib = clamp_contrib(muls(muls(muls(mul(mk(L.e[0], L.e[1], L.e[2]), brdf), geom), sz2), W));
                        ld = l;
                        target_vid = L.vid;
                        have = true;
                    }
                }
            }
        }
        if (res.m > 0u) em.records.push_back(ResRecord{primary_vid, slot, res});
    } else {
        float wsum = 0.0f, chosen_t = 0.0f;
        uint32_t chosen = 0u;
        for (int k = 0; k < 4; k++) {
            uint32_t pick = uint32_t(rand01(rng) * float(n_lights));
            if (pick >= n_lights) pick = n_lights - 1u;
            const EmLight& cand = lights[pick];
            const float lum = gmax(luminance(cand.e), 1e-6f);
            const float target = lum * float(cand.size * cand.size);
            wsum += target;
            if (rand01(rng) * wsum < target) {
                chosen = pick;
                chosen_t = target;
            }
        }
        const float avg_t = wsum / 4.0f;
        const EmLight& L = lights[chosen];
        uint32_t face = uint32_t(rand01(rng) * 6.0f);
        if (face >= 6u) face = 5u;
        f3 fn, ft, fb;
        face_frame(face, fn, ft, fb);
        const float u1 = rand01(rng);
        const float u2 = rand01(rng);
        const f3 lp = face_point(L, fn, ft, fb, u1, u2);
        f3 l = sub(lp, sp);
        const float d2 = dot(l, l);
        const float dist = std::sqrt(d2);
        if (dist > 1e-3f && chosen_t > 0.0f) {
            l = divs(l, dist);
            const float cx = gmax(dot(N, l), 0.0f);
            const float cy = gmax(dot(mk(-l.x, -l.y, -l.z), fn), 0.0f);
            if (cx > 0.0f && cy > 0.0f) {
                const f3 brdf = evaluate_brdf(dir, l, N, albedo, m.roughness, m.metallic, m.specular);
                const float area = 6.0f * float(L.size) * float(L.size);
                const float ris = float(n_lights) * avg_t / gmax(chosen_t, 1e-6f);
                const float geom = cy / gmax(d2, 1e-6f);
                contrib = clamp_contrib(muls(muls(muls(mul(mk(L.e[0], L.e[1], L.e[2]), brdf), geom), area), ris));
                ld = l;
                target_vid = L.vid;
                have = true;
            }
        }
    }
    if (!have) return;
    const Hit sh = raycast(s, sp, ld, P.bounce_controlchecks, rc);
    st->rays_shadow++;
    em.nee++;
    if (sh.status == ST_HIT && voxel_key(sh.pos) + 1u == target_vid) {
        const f3 w = mul(tp, contrib);
        if (b == 0) direct = add(direct, w); else indirect = add(indirect, w);
    }
}

// The per-pixel plain method: one path of the bounce/shade loop
// (shade.comp:543-575, 838-908) from a known primary hit, with the sun
// next-event estimate in the place of the emissive NEE (shade.comp:631-836 is
// dormant in scenes without emissive voxels).
void trace_path(const Scene& s, const Material* mats, uint32_t n_mats, const ov_frame_params& P,
                const Hit& primary, f3 primary_dir, uint32_t pix_index, uint32_t list_idx, PathOut* out,
                ov_stats* st, RayCounters* rc, EmFrame* em = nullptr, bool shared_sun0 = false) {
    const uint32_t max_bounces = P.bounces + 1u;  // MAX_BOUNCES (wavefront.glsl:23)
    // emit.comp:171-174; list_idx is pixel * spp + sample in the per-pixel
    // method and the shade-list index in the scheduled one
    const uint32_t sample_idx = P.frame_index + pix_index * 2654435761u + list_idx * 1442695040u;
    uint32_t rng = (sample_idx << 8) & 0xFFFFFF00u;
    f3 tp = mk(1, 1, 1);
    f3 dir = primary_dir;
    f3 direct = mk(0, 0, 0), indirect = mk(0, 0, 0);
    Hit hit = primary;
    const f3 sun = mk(P.sun_dir[0], P.sun_dir[1], P.sun_dir[2]);
    const f3 sky = mk(P.sky[0], P.sky[1], P.sky[2]);
    uint32_t b = 0;
    for (;;) {
        if (hit.status != ST_HIT) {  // shade.comp:558-564 (sky in place of the cubemap)
            indirect = add(indirect, mul(sky, tp));
            break;
        }
        const uint32_t mi = hit.material < n_mats ? hit.material : 0u;
        const Material& m = mats[mi];
        const f3 albedo = mk(m.color[0], m.color[1], m.color[2]);
        const f3 N = shading_normal(s, s.fetch(hit.id), dir);
        if (m.emissive) {  // shade.comp:576-583
            const float k = m.emissive_intensity;
            f3 e = mul(mk(albedo.x * k, albedo.y * k, albedo.z * k), tp);
            e = mk(gmin(e.x, 20.0f), gmin(e.y, 20.0f), gmin(e.z, 20.0f));
            if (b == 0) direct = add(direct, e); else indirect = add(indirect, e);
            if (em && b == 0)  // a light seen by a primary ray (shade.comp:585-613)
                em->staged.push_back(EmLight{{albedo.x * k, albedo.y * k, albedo.z * k}, voxel_key(hit.pos) + 1u,
                                             {hit.pos[0], hit.pos[1], hit.pos[2]}, 1u});
        }
        const f3 hit_pos = mk(float(hit.pos[0]), float(hit.pos[1]), float(hit.pos[2]));
        const f3 shading_point = add(add(hit_pos, mk(0.5f, 0.5f, 0.5f)), N);  // shade.comp:635, 892
        if (em) {
            if (!m.emissive && b < 2u)
                emissive_nee(s, P, *em, list_idx, voxel_key(primary.pos) + 1u, b, hit, N, shading_point, dir, tp,
                             albedo, m, rng, direct, indirect, st, rc);
        } else if (!m.emissive && b < 2u && dot(N, sun) > 0.0f) {
            // NEE gate of shade.comp:631 (non-emissive surface, bounce < 2),
            // with the sun's cosine test of shade.comp:811-815
            // shared_sun0: a pixel's later sample, whose first shadow ray is
            // sample 0's (the same origin and direction): its walk is not
            // counted again (the device traces it once)
            const Hit sh = raycast(s, shading_point, sun, P.bounce_controlchecks, (b == 0 && shared_sun0) ? nullptr : rc);
            st->rays_shadow++;
            if (b == 0 && shared_sun0) st->shadow_shared++;
            if (sh.status == ST_ESCAPED) {
                const f3 brdf = evaluate_brdf(dir, sun, N, albedo, m.roughness, m.metallic, m.specular);
                f3 c = muls(brdf, P.sun_intensity);
                c = mk(gmin(c.x, 20.0f), gmin(c.y, 20.0f), gmin(c.z, 20.0f));
                const f3 w = mul(tp, c);
                if (b == 0) direct = add(direct, w); else indirect = add(indirect, w);
            }
        }
        if (b + 1u >= max_bounces) break;  // shade.comp:840-845
        // BRDF sample (shade.comp:850-873)
        const bool use_ggx = m.metallic * (1.0f - m.roughness) > 0.5f;
        f3 sdir, bt;
        if (use_ggx) {
            const f3 V = mk(-dir.x, -dir.y, -dir.z);
            const f3 H = sample_ggx_vndf(N, V, m.roughness, rng);
            sdir = reflect(dir, H);
            if (dot(sdir, N) <= 0.0f) {
                sdir = cosine_direction(N, rng);
                bt = evaluate_brdf(dir, sdir, N, albedo, m.roughness, m.metallic, m.specular);
            } else {
                const f3 F0 = mk(0.04f * (1.0f - m.metallic) + albedo.x * m.metallic,
                                 0.04f * (1.0f - m.metallic) + albedo.y * m.metallic,
                                 0.04f * (1.0f - m.metallic) + albedo.z * m.metallic);
                bt = ggx_throughput(N, V, sdir, H, m.roughness, F0);
            }
        } else {
            sdir = cosine_direction(N, rng);
            bt = evaluate_brdf(dir, sdir, N, albedo, m.roughness, m.metallic, m.specular);
        }
        f3 ntp = mul(tp, bt);
        // Russian roulette (shade.comp:879-889), RR_START_BOUNCE = 2
        if (b + 1u >= 2u) {
            const float p = gclamp(gmax(ntp.x, gmax(ntp.y, ntp.z)), 0.05f, 0.95f);
            const float xi = rand01(rng);
            if (xi > p) break;
            ntp = divs(ntp, p);
        }
        // survivor (shade.comp:892-895) + trace.comp
        tp = ntp;
        dir = sdir;
        b++;
        hit = raycast(s, shading_point, sdir, P.bounce_controlchecks, rc, true);
        st->rays_bounce++;
    }
    out->direct = direct;
    out->indirect = indirect;
}

// Deposit value: the reference quantises each channel with
// clamp(rgb, 0, 1024) (packRgbL2, shade.comp:154-160); the FP cache keeps the
// clamped channels as floats, direct + indirect summed.
inline void deposit_value(const PathOut& p, float out[3]) {
    const float dv[3] = {p.direct.x, p.direct.y, p.direct.z};
    const float iv[3] = {p.indirect.x, p.indirect.y, p.indirect.z};
    for (int c = 0; c < 3; c++) {
        float a = dv[c], b = iv[c];
        if (!(a == a)) a = 0.0f;
        if (!(b == b)) b = 0.0f;
        out[c] = gclamp(a, 0.0f, 1024.0f) + gclamp(b, 0.0f, 1024.0f);
    }
}

// The two channels of a deposit apart (packRgbL2 of each, shade.comp:162-167).
inline void deposit_dual(const PathOut& p, float d[3], float e[3]) {
    const float dv[3] = {p.direct.x, p.direct.y, p.direct.z};
    const float iv[3] = {p.indirect.x, p.indirect.y, p.indirect.z};
    for (int c = 0; c < 3; c++) {
        float a = dv[c], b = iv[c];
        if (!(a == a)) a = 0.0f;
        if (!(b == b)) b = 0.0f;
        d[c] = gclamp(a, 0.0f, 1024.0f) + 0.0f;
        e[c] = 0.0f + gclamp(b, 0.0f, 1024.0f);
    }
}

// ---------------------------------------------------------------------------
// The reference's dual-channel lBuffer (shade.comp:96-257 depositSampleDual,
// resolve.comp:109-148 lookupVoxelAvg, rank.comp:66-87), rows of 32 slots x
// 12 words, applied sequentially in (row, path slot) order per frame.
// ---------------------------------------------------------------------------
constexpr uint32_t kFrameLbuffer = 256;  // VE_FRAME_LBUFFER
constexpr uint32_t kLbWidth = 32768, kLbSlots = 32, kLbStride = 12, kLbRowWords = kLbSlots * kLbStride;
inline uint32_t lb_row(uint32_t vid) { return vid % (kLbWidth - 1u) + 1u; }
inline void lb_pack(const float c[3], uint32_t out[4]) {  // packRgbL2 (shade.comp:154-160)
    for (int k = 0; k < 3; k++) out[k] = uint32_t(gclamp(c[k], 0.0f, 1024.0f) * 255.0f);
    const uint32_t L = (out[0] + out[1] + out[2]) / 3u;
    out[3] = L * L;
}
inline void lb_reset(uint32_t* s, uint32_t vid, const uint32_t d[4], const uint32_t e[4], uint32_t time) {
    s[0] = vid;
    s[1] = 1u; s[2] = d[0]; s[3] = d[1]; s[4] = d[2]; s[5] = d[3];
    s[6] = 1u; s[7] = e[0]; s[8] = e[1]; s[9] = e[2]; s[10] = e[3];
    s[11] = time;
}
inline void lb_firefly(const uint32_t* s, uint32_t c[4], const ov_frame_params& P) {  // s: the channel's count
    const uint32_t n = s[0];
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
void lb_deposit(uint32_t* row, uint32_t vid, const float dir[3], const float ind[3], const ov_frame_params& P) {
    uint32_t d[4], e[4];
    lb_pack(dir, d);
    lb_pack(ind, e);
    uint32_t cand_t = 0xFFFFFFFFu, cand_i = 0u;
    for (uint32_t i = 0; i < kLbSlots; i++) {
        uint32_t* s = row + i * kLbStride;
        if (s[0] == 0u) s[0] = vid;
        const uint32_t id = s[0], t = s[11];
        if (id != vid) {
            if (t < cand_t) {
                cand_t = t;
                cand_i = i;
            }
            continue;
        }
        if (!P.disable_stale_reset && t != 0u && t + P.update_time < P.time) {
            lb_reset(s, vid, d, e, P.time);
            return;
        }
        if (s[1] >= P.sample_cap_direct)
            for (int k = 1; k <= 5; k++) s[k] >>= 1;
        if (s[6] >= P.sample_cap_indirect)
            for (int k = 6; k <= 10; k++) s[k] >>= 1;
        lb_firefly(s + 1, d, P);
        lb_firefly(s + 6, e, P);
        s[1] += 1u; s[2] += d[0]; s[3] += d[1]; s[4] += d[2]; s[5] += d[3];
        s[6] += 1u; s[7] += e[0]; s[8] += e[1]; s[9] += e[2]; s[10] += e[3];
        s[11] = P.time;
        return;
    }
    if (cand_t != 0xFFFFFFFFu) lb_reset(row + cand_i * kLbStride, vid, d, e, P.time);
}

// lookupVoxelAvg (resolve.comp:109-148) over the FP64 cache.
struct Avg {
    double rgb[3];
    uint64_t count;
    double var;
};
Avg lookup_avg(const Cache& c, uint32_t vid) {
    Avg a{{0, 0, 0}, 0, 0};
    if (vid == 0) return a;
    const CacheEntry* ep = c.find(vid);
    if (!ep) return a;
    const CacheEntry& e = *ep;
    a.count = e.count;
    if (e.count == 0 || e.weight <= 0.0) return a;
    const double inv = 1.0 / e.weight;
    a.rgb[0] = e.r * inv; a.rgb[1] = e.g * inv; a.rgb[2] = e.b * inv;
    const double meanL = (e.r + e.g + e.b) * inv / 3.0;
    a.var = std::max(e.l2 * inv - meanL * meanL, 0.0);
    return a;
}

// lookupVoxelAvg (resolve.comp:109-148) over the lBuffer, in the device's
// float operations.
Avg lb_lookup(const std::vector<uint32_t>& lb, uint32_t vid) {
    Avg a{{0, 0, 0}, 0, 0};
    if (vid == 0 || lb.empty()) return a;
    const uint32_t* row = lb.data() + size_t(lb_row(vid)) * kLbRowWords;
    for (uint32_t i = 0; i < kLbSlots; i++) {
        const uint32_t* s = row + i * kLbStride;
        if (s[0] != vid) continue;
        const uint32_t dc = s[1], ic = s[6];
        a.count = uint64_t(dc) + ic;
        if (dc + ic == 0u) return a;
        float da[3] = {0, 0, 0}, ia[3] = {0, 0, 0};
        float var = 0.0f;
        if (dc > 0u) {
            const float inv = 1.0f / float(dc);
            for (int k = 0; k < 3; k++) da[k] = float(s[2 + k]) * inv / 255.0f;
        }
        if (ic > 0u) {
            const float inv = 1.0f / float(ic);
            for (int k = 0; k < 3; k++) ia[k] = float(s[7 + k]) * inv / 255.0f;
            const float meanL = float(s[7] + s[8] + s[9]) * inv / 3.0f;
            var = gmax(float(s[10]) * inv - meanL * meanL, 0.0f) / (255.0f * 255.0f);
        }
        for (int k = 0; k < 3; k++) a.rgb[k] = double(da[k] + ia[k]);
        a.count = uint32_t(dc + ic);
        a.var = double(var);
        return a;
    }
    return a;
}
// lookupIndirectVariance (rank.comp:66-87), raw quantised units.
float lb_indirect_variance(const std::vector<uint32_t>& lb, uint32_t vid) {
    if (lb.empty()) return 0.0f;
    const uint32_t* row = lb.data() + size_t(lb_row(vid)) * kLbRowWords;
    for (uint32_t i = 0; i < kLbSlots; i++) {
        const uint32_t* s = row + i * kLbStride;
        if (s[0] == 0u) return 0.0f;
        if (s[0] != vid) continue;
        const uint32_t c = s[6];
        if (c < 2u) return 0.0f;
        const float fc = float(c);
        const float meanL = float(s[7] + s[8] + s[9]) / (3.0f * fc);
        const float meanL2 = float(s[10]) / fc;
        return gmax(meanL2 - meanL * meanL, 0.0f);
    }
    return 0.0f;
}

inline double aces(double x) {  // final.frag:11-18
    double v = (x * (2.51 * x + 0.03)) / (x * (2.43 * x + 0.59) + 0.14);
    return v < 0.0 ? 0.0 : (v > 1.0 ? 1.0 : v);
}

// Scheduling thresholds carried from frame to frame (threshold.comp's
// output, read by the next frame's rank.comp): +inf / -inf before the first
// scheduled frame, which puts every voxel in the middle tier.
struct Renderer {
    Cache cache;
    float t_high = std::numeric_limits<float>::infinity();
    float t_mid = -std::numeric_limits<float>::infinity();
    // emissive frames: the light registry, the vids it has claimed (kept or
    // dropped at capacity) and the committed per-voxel reservoirs
    std::vector<EmLight> lights;
    std::unordered_set<uint32_t> em_claimed;
    std::unordered_map<uint32_t, Reservoir> res;
    std::vector<uint32_t> lb;  // lBuffer frames: kLbWidth rows x 32 slots x 12 words
    std::vector<uint32_t> ncodes;  // ball-normal scenes: the code table their leaf words index
    Avg lookup(bool lbm, uint32_t vid) const { return lbm ? lb_lookup(lb, vid) : lookup_avg(cache, vid); }
};

// End of an emissive frame: new lights in vid order fill the registry up to
// its capacity (all of them stay claimed); each voxel keeps the reservoir of
// its largest path slot.
void commit_emissive(Renderer* R, std::vector<EmFrame>& ems, ov_stats* total) {
    std::vector<EmLight> fresh;
    for (auto& em : ems)
        for (const EmLight& L : em.staged)
            if (R->em_claimed.insert(L.vid).second) fresh.push_back(L);
    std::sort(fresh.begin(), fresh.end(), [](const EmLight& a, const EmLight& b) { return a.vid < b.vid; });
    for (const EmLight& L : fresh)
        if (R->lights.size() < kEmCapacity) R->lights.push_back(L);
    std::unordered_map<uint32_t, const ResRecord*> win;
    for (auto& em : ems)
        for (const ResRecord& r : em.records) {
            auto it = win.find(r.vid);
            if (it == win.end() || it->second->slot < r.slot) win[r.vid] = &r;
        }
    for (auto& kv : win) R->res[kv.first] = kv.second->r;
    total->emissive_lights = R->lights.size();
    total->restir_commits = win.size();
    for (auto& em : ems) total->nee_emissive += em.nee;
}

constexpr uint32_t kRankBins = 256;
constexpr uint32_t kFrameScheduled = 64;  // VE_FRAME_SCHEDULED

inline f3 pixel_dir(const float cam[16], uint32_t px, uint32_t py, uint32_t W, uint32_t H) {
    // generate_primary.comp:44-52
    const f3 plane = mk(cam[4], cam[5], cam[6]);
    const f3 right = mk(cam[8], cam[9], cam[10]);
    const f3 up = mk(cam[12], cam[13], cam[14]);
    const float ndx = (float(px) + 0.5f) / float(W) * 2.0f - 1.0f;
    const float ndy = (float(py) + 0.5f) / float(H) * 2.0f - 1.0f;
    return normalize(sub(add(plane, muls(right, ndx)), muls(up, ndy)));
}

// One scheduled frame's paths (schedule.comp, rank.comp, threshold.comp,
// emit.comp), written as sequential loops over pixels:
//   schedule  every hit pixel claims its voxel; the voxel keeps its pixel
//             count and its smallest pixel index (the representative)
//   rank      importance = w_pix * clamp(pixels / pixels_norm)
//                        + w_var * clamp(var * 255^2 / variance_norm)
//             (var: the cache's luminance variance, 0 below two samples);
//             2 paths at or above t_high, 1 at or above t_mid, else
//             min_samples; a 256-bin histogram of the importances
//   list      entries {vid, pixel} in representative-pixel order starting
//             at pixel (frame * 0x9E3779B9 mod 2^32) mod pixels and wrapping,
//             cut at min(shading_budget, 2 * pixels)
//   threshold the next frame's t_high / t_mid: the bins where the reverse
//             cumulative count reaches top_fraction and top + mid fractions
//   emit      one path per entry from the representative pixel's primary
//             hit, the entry index seeding the path.
// The device implementation follows the same deterministic order (smallest
// pixel as the representative, list ordered by rotated pixel); the reference
// keeps the first pixel to claim and appends with atomics, so its budget cut
// falls on whichever voxels rank last in that frame's workgroup order.
void schedule_frame(Renderer* R, const Scene& s, const Material* mats, uint32_t n_mats, const float cam[16],
                    const ov_frame_params* P, uint32_t threads, const std::vector<Hit>& hits,
                    const std::vector<uint32_t>& vids, float* path_rgb,
                    std::vector<std::vector<std::vector<Deposit>>>& deps, std::vector<ov_stats>& tstats,
                    std::vector<RayCounters>& trc, std::vector<EmFrame>& ems) {
    const uint32_t W = P->width, H = P->height, npix = W * H;
    struct Claim { uint32_t pix, count; };
    std::unordered_map<uint32_t, Claim> claims;
    for (uint32_t pix = 0; pix < npix; pix++) {
        const uint32_t vid = vids[pix];
        if (!vid) continue;
        auto it = claims.find(vid);
        if (it == claims.end()) claims.emplace(vid, Claim{pix, 1u});
        else it->second.count++;
    }
    std::vector<uint32_t> hist(kRankBins, 0u);
    std::vector<std::pair<uint32_t, uint32_t>> list;  // {vid, pixel}
    const uint64_t cap = std::min<uint64_t>(P->shading_budget, 2ull * npix);
    const uint32_t rot = uint32_t(uint64_t(P->frame_index * 0x9E3779B9u) % npix);
    uint64_t nvox = 0;
    for (uint32_t j = 0; j < npix; j++) {
        const uint32_t pix = (j + rot) % npix;
        const uint32_t vid = vids[pix];
        if (!vid) continue;
        const Claim& cl = claims[vid];
        if (cl.pix != pix) continue;
        nvox++;
        const float pn = gclamp(float(cl.count) / gmax(P->pixels_norm, 1.0f), 0.0f, 1.0f);
        float vn;
        if (P->flags & kFrameLbuffer) {  // rank.comp:107 on the lBuffer's own scale
            vn = gclamp(lb_indirect_variance(R->lb, vid) / gmax(P->variance_norm, 1.0f), 0.0f, 1.0f);
        } else {
            const Avg a = lookup_avg(R->cache, vid);
            const float var = a.count >= 2u ? float(a.var) : 0.0f;
            vn = gclamp(var * (255.0f * 255.0f) / gmax(P->variance_norm, 1.0f), 0.0f, 1.0f);
        }
        const float imp = P->weight_pixels * pn + P->weight_variance * vn;
        const uint32_t n = imp >= R->t_high ? 2u : (imp >= R->t_mid ? 1u : P->min_samples);
        uint32_t bin = uint32_t(imp * float(kRankBins));
        if (bin >= kRankBins) bin = kRankBins - 1u;
        hist[bin]++;
        for (uint32_t j = 0; j < n && list.size() < cap; j++) list.emplace_back(vid, pix);
    }
    // threshold.comp
    uint32_t total = 0;
    for (uint32_t b = 0; b < kRankBins; b++) total += hist[b];
    if (total == 0u) {
        R->t_high = std::numeric_limits<float>::infinity();
        R->t_mid = -std::numeric_limits<float>::infinity();
    } else {
        const float top = gclamp(P->top_fraction, 0.0f, 1.0f);
        const float mid = gclamp(P->mid_fraction, 0.0f, 1.0f - top);
        const uint32_t top_n = uint32_t(top * float(total)), topmid_n = uint32_t((top + mid) * float(total));
        uint32_t cum = 0, hb = kRankBins, mb = kRankBins;
        for (int b = int(kRankBins) - 1; b >= 0; b--) {
            cum += hist[b];
            if (hb == kRankBins && cum >= top_n) hb = uint32_t(b);
            if (mb == kRankBins && cum >= topmid_n) mb = uint32_t(b);
        }
        if (hb == kRankBins) hb = kRankBins - 1u;
        if (mb == kRankBins) mb = kRankBins - 1u;
        R->t_high = float(hb) / float(kRankBins);
        R->t_mid = float(mb) / float(kRankBins);
    }
    tstats[0].scheduled_voxels += nvox;
    tstats[0].scheduled_paths += list.size();
    // emit + bounce loop, entries interleaved over threads
    auto work = [&](uint32_t t) {
        ov_stats& st = tstats[t];
        for (size_t i = t; i < list.size(); i += threads) {
            const uint32_t vid = list[i].first, pix = list[i].second;
            const f3 dir = pixel_dir(cam, pix % W, pix / W, W, H);
            PathOut po;
            trace_path(s, mats, n_mats, *P, hits[pix], dir, pix, uint32_t(i), &po, &st, &trc[t],
                       ems.empty() ? nullptr : &ems[t]);
            st.paths++;
            Deposit dp;
            dp.vid = vid;
            deposit_value(po, dp.rgb);
            dp.slot = uint32_t(i);
            deposit_dual(po, dp.d, dp.e);
            if (path_rgb) {
                float* o = path_rgb + 3 * uint64_t(i);
                o[0] = dp.rgb[0]; o[1] = dp.rgb[1]; o[2] = dp.rgb[2];
            }
            deps[t][shard_of(vid)].push_back(dp);
        }
    };
    if (threads == 1) {
        work(0);
    } else {
        std::vector<std::thread> th;
        for (uint32_t t = 0; t < threads; t++) th.emplace_back(work, t);
        for (auto& x : th) x.join();
    }
}

}  // namespace

// ===========================================================================
// C API (ctypes)
// ===========================================================================
extern "C" {

uint32_t oracle_version() { return 3u; }

// Builds the reference layout from a voxel list (x, y, z, material) by
// OctreeCPU::insert order then Octree::set.  Returns the word count
// (== size) and writes up to `cap` words.
uint64_t oracle_build(uint32_t depth, const uint32_t* xyzm, uint64_t n, uint32_t* out, uint64_t cap,
                      uint32_t* nvox) {
    PTree t(depth);
    for (uint64_t i = 0; i < n; i++) t.insert(xyzm[4 * i], xyzm[4 * i + 1], xyzm[4 * i + 2], xyzm[4 * i + 3]);
    uint32_t size = 0, nv = 0;
    std::vector<uint32_t> d = t.linearize(&size, &nv);
    const uint64_t m = std::min<uint64_t>(d.size(), cap);
    if (out) std::memcpy(out, d.data(), m * 4);
    if (nvox) *nvox = nv;
    return d.size();
}

// normal.comp restated over the 3x3x3 neighbourhood; writes the normal field
// into every leaf word of `words` (in place).  Leaves are found by walking
// the tree from the root.  mode 0: every neighbour occupancy by a tree
// descent (lookupOccupied, normal.comp:55-70); mode 1: the same occupancy
// read from a bitmask of all leaves (identical on valid trees, fast enough
// for depth-10 scenes), with `threads` workers.
void oracle_fill_normals_mode(uint32_t* words, uint64_t n, uint32_t depth, int mode, uint32_t threads) {
    std::vector<uint32_t> copy(words, words + n);
    Scene s{copy.data(), n, depth};
    const uint32_t L = 1u << depth;
    struct E { uint32_t off, level, x, y, z; };
    std::vector<E> leaves;
    std::vector<E> st;
    // from the root word (slot 0) through its child pointer, as every
    // descent reads it (Octree::set puts the root's children at slots 1..8)
    st.push_back({0u, 0u, 0u, 0u, 0u});
    while (!st.empty()) {
        E e = st.back();
        st.pop_back();
        const uint32_t raw = s.fetch(e.off);
        if (raw & 1u) {
            if (e.level >= depth) continue;
            const uint32_t next = node_next(raw);
            const uint32_t half = L >> (e.level + 1);
            for (uint32_t i = 0; i < 8; i++)
                st.push_back({next + i, e.level + 1, e.x + ((i & 4) ? half : 0u), e.y + ((i & 2) ? half : 0u),
                              e.z + ((i & 1) ? half : 0u)});
        } else if (node_material(raw) != 0u && e.level == depth) {
            leaves.push_back(e);
        }
    }
    std::vector<uint64_t> bits;
    if (mode == 1) {
        bits.assign(((uint64_t(1) << (3 * depth)) + 63) / 64, 0ull);
        for (const E& e : leaves) {
            const uint64_t b = ((uint64_t(e.z) << depth | e.y) << depth) | e.x;
            bits[b >> 6] |= 1ull << (b & 63);
        }
    }
    auto occupied = [&](int64_t x, int64_t y, int64_t z) {
        if (mode == 0) return lookup_occupied(s, x, y, z);
        if (x < 0 || y < 0 || z < 0 || x >= L || y >= L || z >= L) return false;
        const uint64_t b = ((uint64_t(z) << depth | uint64_t(y)) << depth) | uint64_t(x);
        return bool((bits[b >> 6] >> (b & 63)) & 1u);
    };
    auto work = [&](size_t lo, size_t hi) {
        for (size_t i = lo; i < hi; i++) {
            const E& e = leaves[i];
            int ax = 0, ay = 0, az = 0;
            for (int dx = -1; dx <= 1; dx++)
                for (int dy = -1; dy <= 1; dy++)
                    for (int dz = -1; dz <= 1; dz++) {
                        if (dx == 0 && dy == 0 && dz == 0) continue;
                        if (!occupied(int64_t(e.x) + dx, int64_t(e.y) + dy, int64_t(e.z) + dz)) {
                            ax += dx; ay += dy; az += dz;
                        }
                    }
            words[e.off] = (copy[e.off] & 0xFFu) | encode_normal_field(ax, ay, az);
        }
    };
    if (threads <= 1) {
        work(0, leaves.size());
    } else {
        std::vector<std::thread> th;
        for (uint32_t t = 0; t < threads; t++)
            th.emplace_back(work, leaves.size() * t / threads, leaves.size() * (t + 1) / threads);
        for (auto& x : th) x.join();
    }
}

void oracle_fill_normals(uint32_t* words, uint64_t n, uint32_t depth) {
    oracle_fill_normals_mode(words, n, depth, 0, 1);
}

// The reference's own normal mode, normal.comp:55-95 (computeRefinedNormal
// with packNormalAccum): the sum of the offsets d of the EMPTY neighbours
// with 0 < |d|^2 <= R^2 (R = normalPrecision), out-of-volume neighbours
// counted as empty, around the voxel's even-aligned corner — the pass reads
// the position back from the GBuffer's half coordinates times two
// (normal.comp:147-152, generate_primary.comp:73-77); normalize, or (0,1,0)
// when the sum vanishes; 10-10-10 code round((c + 1) * 511).  The codes of all
// leaves, sorted and made unique, form the scene's code table; each leaf's
// normal field (bits 8-30, bit 31 clear) holds its code's index + 1.
// Occupancy by tree descents (lookupOccupied, normal.comp:55-70).  Writes
// the words in place and up to `cap` table codes; returns the table size.
uint64_t oracle_fill_normals_ball(uint32_t* words, uint64_t n, uint32_t depth, uint32_t radius, uint32_t threads,
                                  uint32_t* codes_out, uint64_t cap) {
    std::vector<uint32_t> copy(words, words + n);
    Scene s{copy.data(), n, depth};
    const uint32_t L = 1u << depth;
    struct E { uint32_t off, level, x, y, z; };
    std::vector<E> leaves;
    std::vector<E> st;
    // from the root word (slot 0) through its child pointer, as every
    // descent reads it (Octree::set puts the root's children at slots 1..8)
    st.push_back({0u, 0u, 0u, 0u, 0u});
    while (!st.empty()) {
        E e = st.back();
        st.pop_back();
        const uint32_t raw = s.fetch(e.off);
        if (raw & 1u) {
            if (e.level >= depth) continue;
            const uint32_t next = node_next(raw);
            const uint32_t half = L >> (e.level + 1);
            for (uint32_t i = 0; i < 8; i++)
                st.push_back({next + i, e.level + 1, e.x + ((i & 4) ? half : 0u), e.y + ((i & 2) ? half : 0u),
                              e.z + ((i & 1) ? half : 0u)});
        } else if (node_material(raw) != 0u && e.level == depth) {
            leaves.push_back(e);
        }
    }
    const int R = int(radius);
    std::vector<uint32_t> code(leaves.size());
    auto pack = [](float c) {
        int v = int(std::round((c + 1.0f) * 511.0f));
        v = v < 0 ? 0 : (v > 1022 ? 1022 : v);
        return uint32_t(v);
    };
    auto work = [&](size_t lo, size_t hi) {
        for (size_t i = lo; i < hi; i++) {
            const int64_t px = leaves[i].x & ~1u, py = leaves[i].y & ~1u, pz = leaves[i].z & ~1u;
            int ax = 0, ay = 0, az = 0;
            for (int dx = -R; dx <= R; dx++)
                for (int dy = -R; dy <= R; dy++)
                    for (int dz = -R; dz <= R; dz++) {
                        if (dx == 0 && dy == 0 && dz == 0) continue;
                        if (dx * dx + dy * dy + dz * dz > R * R) continue;
                        if (!lookup_occupied(s, px + dx, py + dy, pz + dz)) {
                            ax += dx; ay += dy; az += dz;
                        }
                    }
            const f3 acc = mk(float(ax), float(ay), float(az));
            const float len = std::sqrt(dot(acc, acc));
            const f3 nv = len > 0.001f ? divs(acc, len) : mk(0.0f, 1.0f, 0.0f);
            code[i] = (pack(nv.x) << 22) | (pack(nv.y) << 12) | (pack(nv.z) << 2);
        }
    };
    if (threads <= 1) {
        work(0, leaves.size());
    } else {
        std::vector<std::thread> th;
        for (uint32_t t = 0; t < threads; t++)
            th.emplace_back(work, leaves.size() * t / threads, leaves.size() * (t + 1) / threads);
        for (auto& x : th) x.join();
    }
    std::vector<uint32_t> table(code);
    std::sort(table.begin(), table.end());
    table.erase(std::unique(table.begin(), table.end()), table.end());
    for (size_t i = 0; i < leaves.size(); i++) {
        const uint32_t idx = uint32_t(std::lower_bound(table.begin(), table.end(), code[i]) - table.begin());
        words[leaves[i].off] = (copy[leaves[i].off] & 0xFFu) | ((idx + 1u) << 8);
    }
    if (codes_out) std::memcpy(codes_out, table.data(), std::min<uint64_t>(cap, table.size()) * 4);
    return table.size();
}

// The code table the next frames' ball-normal leaves index (n = 0: none).
void oracle_renderer_set_normal_codes(void* rp, const uint32_t* codes, uint64_t n) {
    Renderer* R = static_cast<Renderer*>(rp);
    R->ncodes.assign(codes, codes + n);
}

int oracle_lookup_occupied(const uint32_t* words, uint64_t n, uint32_t depth, int64_t x, int64_t y, int64_t z) {
    Scene s{words, n, depth};
    return lookup_occupied(s, x, y, z) ? 1 : 0;
}

// Camera::UpdateUBO (src/renderer/camera.cpp:39-50): ubo = {position,
// cameraPlane = direction, right, up} as 4 x vec4.
void oracle_camera_ubo(const float pos[3], const float dir[3], float fov_deg, float aspect, float ubo[16]) {
    // glm (host) semantics: normalize(v) = v * inversesqrt(dot(v, v))
    auto gnorm = [](f3 v) { return muls(v, 1.0f / std::sqrt(dot(v, v))); };
    const f3 d = mk(dir[0], dir[1], dir[2]);
    const float tn = std::tan((fov_deg / 2.0f) * 0.01745329251994329576923690768489f);
    const f3 right = muls(muls(gnorm(cross(mk(0, 1, 0), d)), tn), aspect);
    const f3 up = muls(gnorm(cross(right, d)), tn);
    const float v[16] = {pos[0], pos[1], pos[2], 0, d.x, d.y, d.z, 0, right.x, right.y, right.z, 0,
                         up.x, up.y, up.z, 0};
    std::memcpy(ubo, v, sizeof(v));
}

// Single ray through the restated DDA.  out = {status, id, material, x, y,
// z, size, checks}; fetch counters accumulate into fetch[2] when non-null.
void oracle_raycast(const uint32_t* words, uint64_t n, uint32_t depth, const float o[3], const float d[3],
                    uint32_t controlchecks, uint32_t out[8], uint64_t fetch[2]) {
    Scene s{words, n, depth};
    RayCounters rc;
    Hit h = raycast(s, mk(o[0], o[1], o[2]), mk(d[0], d[1], d[2]), controlchecks, &rc);
    out[0] = uint32_t(h.status); out[1] = h.id; out[2] = h.material;
    out[3] = h.pos[0]; out[4] = h.pos[1]; out[5] = h.pos[2];
    out[6] = h.size; out[7] = h.checks;
    if (fetch) { fetch[0] += rc.fetch_restart; fetch[1] += rc.fetch_min; }
}

// oracle_raycast over n rays (3 f32 origin / direction per ray, 8 u32 out
// per ray), rays split across `threads` std::threads.
void oracle_raycast_batch(const uint32_t* words, uint64_t n_words, uint32_t depth, const float* o, const float* d,
                          uint64_t n, uint32_t controlchecks, uint32_t threads, uint32_t* out) {
    Scene s{words, n_words, depth};
    if (threads == 0) threads = 1;
    std::vector<std::thread> th;
    for (uint32_t t = 0; t < threads; t++)
        th.emplace_back([&, t] {
            RayCounters rc;
            for (uint64_t i = t; i < n; i += threads) {
                const Hit h = raycast(s, mk(o[3 * i], o[3 * i + 1], o[3 * i + 2]), mk(d[3 * i], d[3 * i + 1], d[3 * i + 2]),
                                      controlchecks, &rc);
                uint32_t* w = out + 8 * i;
                w[0] = uint32_t(h.status); w[1] = h.id; w[2] = h.material;
                w[3] = h.pos[0]; w[4] = h.pos[1]; w[5] = h.pos[2];
                w[6] = h.size; w[7] = h.checks;
            }
        });
    for (auto& x : th) x.join();
}

// The specular lobe's power function, element-wise (pinned in tests against
// float64 pow).
void oracle_pow_unit(const float* x, const float* e, uint64_t n, float* out) {
    for (uint64_t i = 0; i < n; i++) out[i] = pow_unit(x[i], e[i]);
}

uint32_t oracle_voxel_key(uint32_t x, uint32_t y, uint32_t z) {
    const uint32_t p[3] = {x, y, z};
    return voxel_key(p);
}

// Draws `n` values of rand() from `state` (golden RNG vectors).
uint32_t oracle_rand_seq(uint32_t state, uint32_t n, float* out) {
    for (uint32_t i = 0; i < n; i++) out[i] = rand01(state);
    return state;
}

void oracle_sincos_turn(const float* u, uint64_t n, float* s, float* c) {
    for (uint64_t i = 0; i < n; i++) sincos_turn(u[i], &s[i], &c[i]);
}

void oracle_shading_normal(uint32_t leaf_word, const float dir[3], float out[3]) {
    const Scene none{nullptr, 0, 0};
    f3 v = shading_normal(none, leaf_word, mk(dir[0], dir[1], dir[2]));
    out[0] = v.x; out[1] = v.y; out[2] = v.z;
}

void* oracle_renderer_new() { return new Renderer(); }

// depositSampleDual over a caller's table (kLbWidth rows x 32 x 12 words):
// records of 8 words {vid, unused, d.rgb (f32), e.rgb (f32)} applied in the
// given order (pinned in tests against a transcription of the shader).
void oracle_lb_apply(const uint32_t* rec, uint64_t n, const ov_frame_params* P, uint32_t* table) {
    for (uint64_t i = 0; i < n; i++) {
        const uint32_t* r = rec + 8 * i;
        float d[3], e[3];
        std::memcpy(d, r + 2, 12);
        std::memcpy(e, r + 5, 12);
        lb_deposit(table + size_t(lb_row(r[0])) * kLbRowWords, r[0], d, e, *P);
    }
}

// The lBuffer's occupied slots as {row, slot, 12 words} records in (row,
// slot) order (the layout of the product's ve_lbuffer_dump); returns the
// number of occupied slots.
uint64_t oracle_lbuffer_dump(void* rp, uint32_t* out, uint64_t cap) {
    const Renderer* R = static_cast<Renderer*>(rp);
    uint64_t k = 0;
    if (R->lb.empty()) return 0;
    for (uint32_t r = 0; r < kLbWidth; r++)
        for (uint32_t i = 0; i < kLbSlots; i++) {
            const uint32_t* w = R->lb.data() + size_t(r) * kLbRowWords + i * kLbStride;
            if (w[0] == 0u) continue;
            if (out && k < cap) {
                out[14 * k] = r;
                out[14 * k + 1] = i;
                std::memcpy(out + 14 * k + 2, w, kLbStride * 4);
            }
            k++;
        }
    return k;
}
void oracle_renderer_free(void* r) { delete static_cast<Renderer*>(r); }

// Number of cache entries and a dump: vids[i], counts[i], and
// values[5*i..] = {weight, r, g, b, l2} (FP64).
uint64_t oracle_cache_dump(void* rp, uint32_t* vids, uint64_t* counts, double* values, uint64_t cap) {
    Renderer* r = static_cast<Renderer*>(rp);
    uint64_t i = 0;
    std::vector<uint32_t> keys;
    keys.reserve(r->cache.size());
    for (auto& m : r->cache.map)
        for (auto& kv : m) keys.push_back(kv.first);
    std::sort(keys.begin(), keys.end());
    for (uint32_t k : keys) {
        if (i >= cap) break;
        const CacheEntry& e = *r->cache.find(k);
        if (vids) vids[i] = k;
        if (counts) counts[i] = e.count;
        if (values) {
            values[5 * i] = e.weight; values[5 * i + 1] = e.r; values[5 * i + 2] = e.g;
            values[5 * i + 3] = e.b; values[5 * i + 4] = e.l2;
        }
        i++;
    }
    return keys.size();
}

// One frame of the plain method (the four passes of
// Renderer::runWavefrontFrame, renderer.cpp:282-649, in per-pixel form):
//   1 primary DDA per pixel -> GBuffer {checks, material, hit node, vid}
//     (generate_primary.comp:38-85; .z carries the hit-node index)
//   2 spp paths per hit pixel through the bounce/shade loop (trace_path)
//   3 AccumPass: decay then deposit into the FP64 cache (fixed merge order)
//   4 AvgPass + tonemap per pixel (resolve.comp:362-382, final.frag:11-18)
// Rows [row_begin, row_end) are rendered (all rows when row_end == 0) with
// `threads` std::threads, rows interleaved across threads.  gbuf: 4 u32 per
// pixel; rgb, mapped: 3 f32 per pixel (null to skip).  Paths' per-sample
// values are written to `path_rgb` (3 f32 per path, index pix*spp+s) when
// non-null.
int oracle_render_frame(void* rp, const uint32_t* words, uint64_t n_words, uint32_t depth, const void* materials,
                        uint32_t n_mats, const float cam[16], const ov_frame_params* P, uint32_t threads,
                        uint32_t row_begin, uint32_t row_end, uint32_t* gbuf, float* rgb, float* mapped,
                        float* path_rgb, ov_stats* stats_out) {
    Renderer* R = static_cast<Renderer*>(rp);
    Scene s{words, n_words, depth};
    s.ncodes = R->ncodes.data();
    s.n_ncodes = R->ncodes.size();
    scene_clip_box(s);
    const Material* mats = static_cast<const Material*>(materials);
    const uint32_t W = P->width, H = P->height;
    if (row_end == 0 || row_end > H) row_end = H;
    if (row_begin > row_end) row_begin = row_end;
    if (threads == 0) threads = 1;
    const bool sched = (P->flags & kFrameScheduled) != 0;
    if (sched && (row_begin != 0 || row_end != H)) return -1;  // the schedule spans the whole view
    // emissive frames commit lights and reservoirs once per whole frame
    if ((P->flags & kFrameEmissive) && (row_begin != 0 || row_end != H)) return -1;
    std::vector<Hit> hits(sched ? size_t(W) * H : 0);
    std::vector<uint32_t> vids(sched ? size_t(W) * H : 0, 0u);

    const bool lbm = (P->flags & kFrameLbuffer) != 0;
    // temporal decay of the cache before this frame's deposits (the lBuffer
    // has none: its channels halve at their sample caps)
    if (!lbm) run_parallel(kShards, threads, [&](uint32_t sh) {
        for (auto& kv : R->cache.map[sh]) {
            CacheEntry& e = kv.second;
            const double k = P->decay;
            e.weight *= k; e.r *= k; e.g *= k; e.b *= k; e.l2 *= k;
        }
    });

    const f3 cpos = mk(cam[0], cam[1], cam[2]);
    const f3 plane = mk(cam[4], cam[5], cam[6]);
    const f3 right = mk(cam[8], cam[9], cam[10]);
    const f3 up = mk(cam[12], cam[13], cam[14]);

    std::vector<std::vector<std::vector<Deposit>>> deps(threads, std::vector<std::vector<Deposit>>(kShards));
    std::vector<ov_stats> tstats(threads);
    std::vector<RayCounters> trc(threads);
    // emissive frames: the registry and reservoirs as the frame begins
    std::vector<EmFrame> ems((P->flags & kFrameEmissive) ? threads : 0);
    for (auto& em : ems) {
        em.lights = &R->lights;
        em.res = &R->res;
    }
    const uint32_t rows = row_end - row_begin;
    // static interleaved rows (row r -> thread r mod threads): balanced and
    // deterministic; deposits merge in thread order below
    (void)rows;
    auto work = [&](uint32_t t) {
        ov_stats& st = tstats[t];
        std::memset(&st, 0, sizeof(st));
        for (uint32_t py = row_begin + t; py < row_end; py += threads) {
            for (uint32_t px = 0; px < W; px++) {
                // pixel -> ray (generate_primary.comp:44-52)
                const float ndx = (float(px) + 0.5f) / float(W) * 2.0f - 1.0f;
                const float ndy = (float(py) + 0.5f) / float(H) * 2.0f - 1.0f;
                const f3 dir = normalize(sub(add(plane, muls(right, ndx)), muls(up, ndy)));
                const Hit h = raycast(s, cpos, dir, P->primary_controlchecks, &trc[t]);
                st.rays_primary++;
                const uint32_t pix = py * W + px;
                uint32_t vid = 0;
                if (h.status == ST_HIT) vid = voxel_key(h.pos) + 1u;
                if (gbuf) {
                    gbuf[4 * uint64_t(pix) + 0] = h.checks;
                    gbuf[4 * uint64_t(pix) + 1] = h.status == ST_HIT ? h.material : 0u;
                    gbuf[4 * uint64_t(pix) + 2] = h.status == ST_HIT ? h.id : 0u;
                    gbuf[4 * uint64_t(pix) + 3] = vid;
                }
                if (sched) {
                    hits[pix] = h;
                    vids[pix] = vid;
                    continue;
                }
                if (vid == 0) continue;
                for (uint32_t smp = 0; smp < P->spp; smp++) {
                    PathOut po;
                    trace_path(s, mats, n_mats, *P, h, dir, pix, pix * P->spp + smp, &po, &st, &trc[t],
                               ems.empty() ? nullptr : &ems[t], ems.empty() && smp > 0);
                    st.paths++;
                    Deposit dp;
                    dp.vid = vid;
                    deposit_value(po, dp.rgb);
                    dp.slot = pix * P->spp + smp;
                    deposit_dual(po, dp.d, dp.e);
                    if (path_rgb) {
                        float* o = path_rgb + 3 * (uint64_t(pix) * P->spp + smp);
                        o[0] = dp.rgb[0]; o[1] = dp.rgb[1]; o[2] = dp.rgb[2];
                    }
                    deps[t][shard_of(vid)].push_back(dp);
                }
            }
        }
    };
    if (threads == 1) {
        work(0);
    } else {
        std::vector<std::thread> th;
        for (uint32_t t = 0; t < threads; t++) th.emplace_back(work, t);
        for (auto& x : th) x.join();
    }
    if (sched) schedule_frame(R, s, mats, n_mats, cam, P, threads, hits, vids, path_rgb, deps, tstats, trc, ems);
    ov_stats total{};
    for (uint32_t t = 0; t < threads; t++) {
        total.rays_primary += tstats[t].rays_primary;
        total.rays_bounce += tstats[t].rays_bounce;
        total.rays_shadow += tstats[t].rays_shadow;
        total.shadow_shared += tstats[t].shadow_shared;
        total.paths += tstats[t].paths;
        total.fetch_restart += trc[t].fetch_restart;
        total.fetch_min += trc[t].fetch_min;
        total.steps += trc[t].steps;
        total.scheduled_voxels += tstats[t].scheduled_voxels;
        total.scheduled_paths += tstats[t].scheduled_paths;
        for (uint32_t sh = 0; sh < kShards; sh++) total.deposits += deps[t][sh].size();
    }
    if (!ems.empty()) commit_emissive(R, ems, &total);
    if (lbm) {  // AccumPass into the lBuffer: every deposit, in (row, path slot) order
        if (R->lb.empty()) R->lb.assign(size_t(kLbWidth) * kLbRowWords, 0u);
        std::vector<const Deposit*> all;
        for (uint32_t t = 0; t < threads; t++)
            for (uint32_t sh = 0; sh < kShards; sh++)
                for (const Deposit& d : deps[t][sh]) all.push_back(&d);
        std::sort(all.begin(), all.end(), [](const Deposit* x, const Deposit* y) {
            const uint32_t rx = lb_row(x->vid), ry = lb_row(y->vid);
            return rx != ry ? rx < ry : x->slot < y->slot;
        });
        for (const Deposit* d : all) lb_deposit(R->lb.data() + size_t(lb_row(d->vid)) * kLbRowWords, d->vid, d->d, d->e, *P);
    } else run_parallel(kShards, threads, [&](uint32_t sh) {
        auto& m = R->cache.map[sh];
        for (uint32_t t = 0; t < threads; t++)
            for (const Deposit& d : deps[t][sh]) {
                CacheEntry& e = m[d.vid];
                const float Lf = ((d.rgb[0] + d.rgb[1]) + d.rgb[2]) / 3.0f;
                e.count += 1;
                e.weight += 1.0;
                e.r += double(d.rgb[0]); e.g += double(d.rgb[1]); e.b += double(d.rgb[2]);
                e.l2 += double(Lf * Lf);
            }
    });

    // AvgPass (resolve.comp main :362-382 with resolveDefault :224-261,
    // reconstructTimeout :193-219, and the visualisation modes :266-359)
    if (rgb || mapped) {
        const double sky[3] = {P->sky[0], P->sky[1], P->sky[2]};
        auto gb = [&](int64_t x, int64_t y, int k) -> uint32_t {
            if (y < int64_t(row_begin) || y >= int64_t(row_end)) return 0u;
            return gbuf[4 * uint64_t(y * W + x) + k];
        };
        const int dxs[4] = {1, -1, 0, 0}, dys[4] = {0, 0, 1, -1};
        for (uint32_t py = row_begin; py < row_end; py++) {
            for (uint32_t px = 0; px < W; px++) {
                const uint32_t pix = py * W + px;
                const uint32_t checks = gb(px, py, 0), mat = gb(px, py, 1), node = gb(px, py, 2),
                               vid = gb(px, py, 3);
                double col[3] = {0, 0, 0};
                auto reconstruct = [&]() {
                    double sum[3] = {0, 0, 0}, ws = 0;
                    const int R_ = int(P->reconstruction_radius);
                    for (int dy = -R_; dy <= R_; dy++)
                        for (int dx = -R_; dx <= R_; dx++) {
                            if (dx == 0 && dy == 0) continue;
                            const int64_t qx = int64_t(px) + dx, qy = int64_t(py) + dy;
                            if (qx < 0 || qy < 0 || qx >= W || qy >= H) continue;
                            const uint32_t nv = gb(qx, qy, 3), nc = gb(qx, qy, 0);
                            if (nv == 0 || nc >= P->primary_controlchecks) continue;
                            Avg a = R->lookup(lbm, nv);
                            if (a.count == 0) continue;
                            const double dist = double(dx * dx + dy * dy);
                            const double w = double(std::min<uint64_t>(a.count, 32)) / (1.0 + dist * 0.15);
                            for (int c = 0; c < 3; c++) sum[c] += a.rgb[c] * w;
                            ws += w;
                        }
                    if (ws > 0.0001) { for (int c = 0; c < 3; c++) col[c] = sum[c] / ws; }
                    else { for (int c = 0; c < 3; c++) col[c] = sky[c]; }
                };
                auto miss = [&]() {
                    if (checks >= P->primary_controlchecks) reconstruct();
                    else { for (int c = 0; c < 3; c++) col[c] = sky[c]; }
                };
                switch (P->render_type) {
                    case 1:  // STRUCTURE
                        for (int c = 0; c < 3; c++) col[c] = double(float(checks) / 65.0f);
                        break;
                    case 2:  // ALBEDO
                        if (vid == 0) miss();
                        else if (mat != 0 && mat < 127 && mat < n_mats)
                            for (int c = 0; c < 3; c++) col[c] = mats[mat].color[c];
                        break;
                    case 3:  // NORMAL (from the leaf word's normal field)
                        if (vid == 0) miss();
                        else {
                            const uint32_t w = s.fetch(node);
                            if (has_normal(w)) {
                                const f3 nd = mk(0, 0, 1);
                                f3 nn = shading_normal(s, w, nd);
                                col[0] = nn.x * 0.5 + 0.5; col[1] = nn.y * 0.5 + 0.5; col[2] = nn.z * 0.5 + 0.5;
                            }
                        }
                        break;
                    case 4:  // VOXELID
                        if (vid == 0) miss();
                        else {
                            const uint32_t hid = vid - 1u;
                            col[0] = double(float((hid + 1u) % 255u) / 255.0f);
                            col[1] = double(float(((hid + 1u) / 255u) % 255u) / 255.0f);
                            col[2] = double(float(((hid + 1u) / (255u * 255u)) % 255u) / 255.0f);
                        }
                        break;
                    case 5:  // VARIANCE
                        if (vid == 0) miss();
                        else {
                            Avg a = R->lookup(lbm, vid);
                            double v = a.count >= 2 ? a.var : 0.0;
                            double sc = v * (255.0 * 255.0) / std::max<double>(P->variance_norm, 1.0);
                            sc = sc < 0 ? 0 : (sc > 1 ? 1 : sc);
                            for (int c = 0; c < 3; c++) col[c] = sc;
                        }
                        break;
                    default: {  // DEFAULT
                        if (vid == 0) { miss(); break; }
                        Avg a = R->lookup(lbm, vid);
                        if (a.count >= 128 && a.var < 0.02) {
                            for (int c = 0; c < 3; c++) col[c] = a.rgb[c];
                            break;
                        }
                        double sum[3], ws = double(a.count);
                        for (int c = 0; c < 3; c++) sum[c] = a.rgb[c] * double(a.count);
                        for (int k = 0; k < 4; k++) {
                            const int64_t qx = int64_t(px) + dxs[k], qy = int64_t(py) + dys[k];
                            if (qx < 0 || qy < 0 || qx >= W || qy >= H) continue;
                            const uint32_t nv = gb(qx, qy, 3);
                            if (nv == 0 || nv == vid) continue;
                            Avg na = R->lookup(lbm, nv);
                            if (na.count == 0) continue;
                            const double d0 = na.rgb[0] - a.rgb[0], d1 = na.rgb[1] - a.rgb[1],
                                         d2 = na.rgb[2] - a.rgb[2];
                            const double dc = std::sqrt(d0 * d0 + d1 * d1 + d2 * d2);
                            const double wc = std::exp(-dc * 6.0);
                            const double wv = 1.0 / (1.0 + na.var * 32.0);
                            const double w = wc * wv * double(std::min<uint64_t>(na.count, 32));
                            for (int c = 0; c < 3; c++) sum[c] += na.rgb[c] * w;
                            ws += w;
                        }
                        if (ws > 0.0001) for (int c = 0; c < 3; c++) col[c] = sum[c] / ws;
                        break;
                    }
                }
                if (rgb) for (int c = 0; c < 3; c++) rgb[3 * uint64_t(pix) + c] = float(col[c]);
                if (mapped) for (int c = 0; c < 3; c++) mapped[3 * uint64_t(pix) + c] = float(aces(col[c]));
            }
        }
    }
    if (stats_out) *stats_out = total;
    return 0;
}

}  // extern "C"
