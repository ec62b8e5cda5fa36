// ve_device.cuh — device-side arithmetic of the voxel ray pipeline.
//
// Floating-point policy (bit-exact agreement with the CPU oracle): this
// translation unit is compiled with --fmad=false (no contraction), IEEE
// division and square root; every GLSL min/max is written as the explicit
// select glm uses (min(a,b) = (b<a)?b:a, max(a,b) = (a<b)?b:a) so NaN
// behaviour is pinned; the only fused multiply-adds are the explicit
// __fmaf_rn calls of the sin/cos polynomial.
#pragma once
#include <cstdint>

namespace ve {
namespace dev {

struct f3 {
    float x, y, z;
};
__device__ __forceinline__ f3 mk(float x, float y, float z) { return f3{x, y, z}; }
__device__ __forceinline__ f3 add(f3 a, f3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ f3 sub(f3 a, f3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ f3 mul(f3 a, f3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ f3 muls(f3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ f3 divs(f3 a, float s) { return mk(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ float gmin(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float gmax(float a, float b) { return (a < b) ? b : a; }
__device__ __forceinline__ float gclamp(float x, float lo, float hi) { return gmin(gmax(x, lo), hi); }
__device__ __forceinline__ float dot(f3 a, f3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
__device__ __forceinline__ f3 normalize(f3 v) { return divs(v, sqrtf(dot(v, v))); }
__device__ __forceinline__ f3 cross(f3 a, f3 b) {
    return mk(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}

// ---------------------------------------------------------------------------
// node words (reference src/renderer/octree.hpp:16-37, internal.glsl:18)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t locate(uint32_t x, uint32_t y, uint32_t z, uint32_t p2) {
    return (uint32_t((x & p2) != 0u) << 2) | (uint32_t((y & p2) != 0u) << 1) | uint32_t((z & p2) != 0u);
}
__device__ __forceinline__ bool in_bounds(f3 v, float n) {
    return 0.0f <= v.x && v.x <= n && 0.0f <= v.y && v.y <= n && 0.0f <= v.z && v.z <= n;
}

enum : uint32_t { kHit = 0, kEscaped = 1, kTimeout = 2 };

struct Hit {
    uint32_t status;
    uint32_t id, material;
    uint32_t x, y, z;
    uint32_t size;
    uint32_t checks;
};

// hash + voxelKey (internal.glsl:263-291)
__device__ __forceinline__ uint32_t hash32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
__device__ __forceinline__ uint32_t voxel_key(uint32_t x, uint32_t y, uint32_t z) {
    return hash32(x | (y << 10) | (z << 20)) & 0x7FFFFFFFu;
}

// halton + rand (internal.glsl:57-89).
//
// Same values as the loop `f /= b; q = i / b; r += f * (i - q*b); i = q` run
// with a runtime base, computed faster:
//   * the digit loop is instantiated per base so every division is by a
//     compile-time constant (multiply-high + shift);
//   * the scale factors f_k = (((1/b)/b)/...) are the IEEE quotients of that
//     same division sequence, read from a table built once on the host with
//     identical single-precision divisions;
//   * base 2: every partial sum has <= 24 significant bits, so the float sum is
//     exact and equals the bit-reversed low 24 bits of i scaled by 2^-24.
__constant__ float c_halton_f[16][24];

template <uint32_t B>
__device__ __forceinline__ float halton_const(uint32_t i, int row) {
    float r = 0.0f;
#pragma unroll 1
    for (int k = 0; k < 24 && i > 0u; k++) {
        const uint32_t q = i / B;
        r = r + c_halton_f[row][k] * float(i - q * B);
        i = q;
    }
    return r;
}
__device__ __forceinline__ float halton2(uint32_t i) {
    return float(__brev(i) >> 8) * 5.9604644775390625e-8f;  // exact: <= 24 significant bits
}
__device__ __forceinline__ float halton_idx(uint32_t i, uint32_t idx) {
    switch (idx) {
        case 0: return halton2(i);
        case 1: return halton_const<3>(i, 1);
        case 2: return halton_const<5>(i, 2);
        case 3: return halton_const<7>(i, 3);
        case 4: return halton_const<11>(i, 4);
        case 5: return halton_const<13>(i, 5);
        case 6: return halton_const<17>(i, 6);
        case 7: return halton_const<19>(i, 7);
        case 8: return halton_const<23>(i, 8);
        case 9: return halton_const<29>(i, 9);
        case 10: return halton_const<31>(i, 10);
        case 11: return halton_const<37>(i, 11);
        case 12: return halton_const<41>(i, 12);
        case 13: return halton_const<43>(i, 13);
        case 14: return halton_const<47>(i, 14);
        default: return halton_const<53>(i, 15);
    }
}
__device__ __forceinline__ float rand01(uint32_t& state) {
    const uint32_t dim = state & 0xFFu;
    const uint32_t sample_idx = state >> 8;
    state = (sample_idx << 8) | ((dim + 1u) & 0xFFu);
    const uint32_t effective = sample_idx ^ ((dim >> 4) * 0x9E3779B9u);
    return halton_idx(effective, dim & 15u);
}

// sin/cos of 2*pi*u: quadrant reduction then Taylor polynomials of degree
// 11 (sin) and 12 (cos) on [0, pi/2) in Horner form with explicit fma
// (project-written; same constants and operation order as the oracle).
__device__ __forceinline__ void sincos_turn(float u, float* s_out, float* c_out) {
    const float x = u * 4.0f;
    const float qf = floorf(x);
    const int q = int(qf) & 3;
    const float t = (x - qf) * 0x1.921fb6p+0f;
    const float t2 = t * t;
    float ps = __fmaf_rn(t2, -0x1.ae6456p-26f, 0x1.71de3ap-19f);
    ps = __fmaf_rn(t2, ps, -0x1.a01a02p-13f);
    ps = __fmaf_rn(t2, ps, 0x1.111112p-7f);
    ps = __fmaf_rn(t2, ps, -0x1.555556p-3f);
    const float s = __fmaf_rn(t * t2, ps, t);
    float pc = __fmaf_rn(t2, 0x1.1eed8ep-29f, -0x1.27e4fcp-22f);
    pc = __fmaf_rn(t2, pc, 0x1.a01a02p-16f);
    pc = __fmaf_rn(t2, pc, -0x1.6c16c2p-10f);
    pc = __fmaf_rn(t2, pc, 0x1.555556p-5f);
    pc = __fmaf_rn(t2, pc, -0x1p-1f);
    const float c = __fmaf_rn(t2, pc, 1.0f);
    float so, co;
    if (q == 0) { so = s; co = c; }
    else if (q == 1) { so = c; co = -s; }
    else if (q == 2) { so = -s; co = -c; }
    else { so = -c; co = s; }
    *s_out = so;
    *c_out = co;
}

__device__ __forceinline__ f3 uniform_sphere(uint32_t& rng) {
    const float u1 = rand01(rng);
    const float u2 = rand01(rng);
    const float z = 1.0f - 2.0f * u1;
    const float rr = sqrtf(gmax(1.0f - z * z, 0.0f));
    float sn, cs;
    sincos_turn(u2, &sn, &cs);
    return mk(rr * cs, rr * sn, z);
}

// normalize(N + RandomDirection) (reference shade.comp:869)
__device__ __forceinline__ f3 cosine_direction(f3 n, uint32_t& rng) {
    const f3 v = add(n, uniform_sphere(rng));
    const float d2 = dot(v, v);
    if (!(d2 > 1e-12f)) return n;
    return divs(v, sqrtf(d2));
}

// x^e for x in (0, 1] and e > 0 (the specular lobe's pow(NdotH, exponent)),
// project-written so the host and the device agree bit for bit:
// exp2(e * log2 x) with ln of the mantissa m in [sqrt(1/2), sqrt(2)) from
// the series ln m = 2 atanh(s) = 2 (s + s^3/3 + ... + s^13/13),
// s = (m - 1) / (m + 1), and 2^f, f in [-1/2, 1/2], from the Taylor series
// of e^(f ln 2) to degree 8 (explicit fma throughout).  Results below 2^-125
// read as 0.
__device__ __forceinline__ float pow_unit(float x, float e) {
    if (x != x) return x;  // NaN stays NaN
    const uint32_t bits = __float_as_uint(x);
    int ex = int(bits >> 23) - 127;
    float m = __uint_as_float((bits & 0x007FFFFFu) | 0x3F800000u);
    if (m > 1.41421356f) {
        m = m * 0.5f;
        ex += 1;
    }
    const float s = (m - 1.0f) / (m + 1.0f);
    const float s2 = s * s;
    float p = __fmaf_rn(s2, 0.0769230769f, 0.0909090909f);
    p = __fmaf_rn(s2, p, 0.111111111f);
    p = __fmaf_rn(s2, p, 0.142857143f);
    p = __fmaf_rn(s2, p, 0.2f);
    p = __fmaf_rn(s2, p, 0.333333333f);
    const float lnm = 2.0f * __fmaf_rn(s * s2, p, s);
    const float y = e * (float(ex) + lnm * 1.44269504f);
    if (!(y > -125.0f)) return 0.0f;
    const float n = floorf(y + 0.5f);
    const float t = (y - n) * 0.693147181f;
    float q = __fmaf_rn(t, 2.48015873e-5f, 1.98412698e-4f);
    q = __fmaf_rn(t, q, 1.38888889e-3f);
    q = __fmaf_rn(t, q, 8.33333333e-3f);
    q = __fmaf_rn(t, q, 4.16666667e-2f);
    q = __fmaf_rn(t, q, 0.166666667f);
    q = __fmaf_rn(t, q, 0.5f);
    q = __fmaf_rn(t, q, 1.0f);
    q = __fmaf_rn(t, q, 1.0f);
    return __uint_as_float(__float_as_uint(q) + (uint32_t(int(n)) << 23));
}

// EvaluateBRDF (internal.glsl:120-149)
__device__ __forceinline__ f3 evaluate_brdf(f3 V, f3 L, f3 N, f3 albedo, float roughness, float metallic,
                                            float specular_intensity) {
    const float NdotL = gmax(dot(N, L), 0.001f);
    if (NdotL < 0.001f) return mk(0.0f, 0.0f, 0.0f);
    const float rc = gmax(roughness, 0.01f);
    const float spec_exp = 2.0f / (rc * rc);
    const float kS = specular_intensity * metallic;
    const float kD = 1.0f - kS * 0.5f;
    const f3 diffuse = muls(muls(albedo, kD), 0.31831f);
    float sp;
    if (kS != 0.0f) {
        const f3 H = normalize(sub(L, V));
        const float NdotH = gmax(dot(N, H), 0.001f);
        const float spec_norm = (spec_exp + 2.0f) * 0.15915494f;
        sp = (spec_norm * pow_unit(NdotH, spec_exp)) * kS;
    } else {
        // The lobe is multiplied by kS = 0: the product is +0 whenever the
        // half vector is finite, i.e. whenever |L - V|^2 > 0 (N, L, V are
        // finite unit vectors), and NaN otherwise (0/0 in the normalise).
        const f3 lv = sub(L, V);
        sp = dot(lv, lv) > 0.0f ? 0.0f : __int_as_float(0x7fc00000);
    }
    return muls(mk(diffuse.x + sp, diffuse.y + sp, diffuse.z + sp), NdotL);
}

// smithG1GGX / sampleGGXVNDF / ggxThroughput (internal.glsl:165-239)
__device__ __forceinline__ float smith_g1(float NdotX, float a) {
    const float a2 = a * a;
    return 2.0f * NdotX / (NdotX + sqrtf(a2 + (1.0f - a2) * NdotX * NdotX));
}
__device__ __forceinline__ f3 sample_ggx_vndf(f3 N, f3 V, float roughness, uint32_t& rng) {
    const float a = gmax(roughness * roughness, 0.001f);
    const f3 up = fabsf(N.z) < 0.999f ? mk(0.0f, 0.0f, 1.0f) : mk(1.0f, 0.0f, 0.0f);
    const f3 T = normalize(cross(up, N));
    const f3 B = cross(N, T);
    const f3 Vl = mk(dot(V, T), dot(V, B), dot(V, N));
    const f3 Vh = normalize(mk(a * Vl.x, a * Vl.y, Vl.z));
    const float lensq = Vh.x * Vh.x + Vh.y * Vh.y;
    f3 T1;
    if (lensq > 0.0f) {
        const float is = 1.0f / sqrtf(lensq);
        T1 = mk(-Vh.y * is, Vh.x * is, 0.0f);
    } else {
        T1 = mk(1.0f, 0.0f, 0.0f);
    }
    const f3 T2 = cross(Vh, T1);
    const float r1 = rand01(rng);
    const float r2 = rand01(rng);
    const float r = sqrtf(r1);
    float sn, cs;
    sincos_turn(r2, &sn, &cs);
    const float t1 = r * cs;
    float t2 = r * sn;
    const float s = 0.5f * (1.0f + Vh.z);
    t2 = (1.0f - s) * sqrtf(gmax(1.0f - t1 * t1, 0.0f)) + s * t2;
    const float w = sqrtf(gmax(0.0f, 1.0f - t1 * t1 - t2 * t2));
    const f3 Nh = add(add(muls(T1, t1), muls(T2, t2)), muls(Vh, w));
    const f3 Hl = normalize(mk(a * Nh.x, a * Nh.y, gmax(0.0f, Nh.z)));
    return add(add(muls(T, Hl.x), muls(B, Hl.y)), muls(N, Hl.z));
}
__device__ __forceinline__ f3 ggx_throughput(f3 N, f3 V, f3 L, f3 H, float roughness, f3 F0) {
    const float NdotL = gmax(dot(N, L), 0.001f);
    const float VdotH = gmax(dot(V, H), 0.001f);
    const float a = roughness * roughness;
    const float x = 1.0f - VdotH;
    const float x2 = x * x;
    const float x5 = x2 * x2 * x;
    const f3 F = mk(F0.x + (1.0f - F0.x) * x5, F0.y + (1.0f - F0.y) * x5, F0.z + (1.0f - F0.z) * x5);
    return muls(F, smith_g1(NdotL, a));
}
__device__ __forceinline__ f3 reflect(f3 I, f3 N) { return sub(I, muls(N, 2.0f * dot(N, I))); }

// Shading normal from a leaf word: the stored 3x3x3 gradient (bits 8-22, 5-bit
// two's complement per axis, bit 31 = present) -> normalize -> 10-10-10 code
// of packNormalAccum (normal.comp:90-95) -> UnpackNormal (internal.glsl:22-28)
// -> normalize; absent normals use lookupNormal's face fallback
// (shade.comp:271-274).
__device__ __forceinline__ int sext5(uint32_t v) { return (v & 16u) ? int(v) - 32 : int(v); }
__device__ __forceinline__ float sgnf(float v) { return v > 0.0f ? 1.0f : (v < 0.0f ? -1.0f : 0.0f); }
__device__ __forceinline__ uint32_t pack1022(float c) {
    int v = int(roundf((c + 1.0f) * 511.0f));
    v = v < 0 ? 0 : (v > 1022 ? 1022 : v);
    return uint32_t(v);
}
// Shading normals of every stored gradient (19^3 codes), built on the host
// with the same single-precision operations as shading_normal_compute.
__device__ float4 g_normal_table[19 * 19 * 19];

__device__ __forceinline__ f3 shading_normal_compute(uint32_t leaf_word, f3 ray_dir);

// Index + 1 of a leaf's entry in its scene's ball-normal table (the
// reference's normal mode): bits 8-30 of a leaf word whose bit 31 is clear;
// 0 when the leaf has none.
__device__ __forceinline__ uint32_t ball_index(uint32_t leaf_word) {
    return (leaf_word >> 31) ? 0u : (leaf_word >> 8) & 0x7FFFFFu;
}

// `ntab`/`n_ntab`: the scene's ball-normal table (null for a scene in the
// 3x3x3-gradient mode).
__device__ __forceinline__ f3 shading_normal(uint32_t leaf_word, f3 ray_dir, const float4* ntab = nullptr,
                                             uint32_t n_ntab = 0u) {
    const uint32_t bi = ball_index(leaf_word);
    if (ntab && bi != 0u && bi - 1u < n_ntab) {
        const float4 n = __ldg(ntab + (bi - 1u));
        return mk(n.x, n.y, n.z);
    }
    if (leaf_word >> 31) {
        const int ix = sext5((leaf_word >> 8) & 31u), iy = sext5((leaf_word >> 13) & 31u),
                  iz = sext5((leaf_word >> 18) & 31u);
        if (ix >= -9 && ix <= 9 && iy >= -9 && iy <= 9 && iz >= -9 && iz <= 9) {
            const float4 n = __ldg(&g_normal_table[((ix + 9) * 19 + (iy + 9)) * 19 + (iz + 9)]);
            return mk(n.x, n.y, n.z);
        }
    }
    return shading_normal_compute(leaf_word, ray_dir);
}

__device__ __forceinline__ f3 shading_normal_compute(uint32_t leaf_word, f3 ray_dir) {
    if (!(leaf_word >> 31)) {
        const float ax = fabsf(ray_dir.x), ay = fabsf(ray_dir.y), az = fabsf(ray_dir.z);
        if (ax > ay && ax > az) return mk(-sgnf(ray_dir.x), 0.0f, 0.0f);
        if (ay > az) return mk(0.0f, -sgnf(ray_dir.y), 0.0f);
        return mk(0.0f, 0.0f, -sgnf(ray_dir.z));
    }
    const f3 acc = mk(float(sext5((leaf_word >> 8) & 31u)), float(sext5((leaf_word >> 13) & 31u)),
                      float(sext5((leaf_word >> 18) & 31u)));
    const float len = sqrtf(dot(acc, acc));
    const f3 n = len > 0.001f ? divs(acc, len) : mk(0.0f, 1.0f, 0.0f);
    const f3 u = mk(float(pack1022(n.x)) / 511.0f - 1.0f, float(pack1022(n.y)) / 511.0f - 1.0f,
                    float(pack1022(n.z)) / 511.0f - 1.0f);
    return normalize(u);
}
__device__ __forceinline__ uint32_t encode_normal_field(int ix, int iy, int iz) {
    return ((uint32_t(ix) & 31u) << 8) | ((uint32_t(iy) & 31u) << 13) | ((uint32_t(iz) & 31u) << 18) | (1u << 31);
}

}  // namespace dev
}  // namespace ve
