// raycast.cuh — the octree DDA on the device.
//
// Result-identical to the reference's restart-from-root Raycast /
// RaycastCounted (internal.glsl:297-400): the same slab arithmetic, the same
// step counting (entry intersection counts one check, loop test
// `q++ <= controlchecks`), the same out-of-range-reads-zero rule.  What
// differs is how the descent finds the terminal cell of a DDA step:
//
//   The node read at descent level k depends only on the bits D..D-k of the
//   integer position.  Consecutive DDA positions share their high bits, so a
//   descent restarts at the first level whose bits changed, reusing the
//   child-block offsets `base[k]` the previous descent recorded.  When the
//   new position lies in the previous terminal (empty) cell the previous
//   result is reused outright.  The node words read per ray are then the
//   distinct nodes along its walk instead of (depth+1) per step.
//
//   A descent that restarts above level T0 reads one word of the scene's
//   top table instead of levels 0..T0-1: per cell of the level-(T0-1)
//   grid, the child-block offset reached at level T0, or the terminal level
//   when the cell is empty higher up (built from the node words by
//   k_build_top, bit-identical to walking them).  This shortens the longest
//   descents of a warp — those that cross a coarse cell boundary — which set
//   its lock-step cost.  Fetch-counting runs (COUNT) walk every level.
//
//   Where the table reaches the leaves (T0 = D, every scene of depth 3..10),
//   a restart below level D is one table word and then the leaf word, so the
//   only offset a ray keeps across steps is its leaf block's: the FLAT walk
//   holds it in a register instead of the per-level array in local memory
//   (trace 1.023 -> 0.998 ms, primary 0.398 -> 0.387 ms per 1080p depth-10
//   frame).  Positions with a coordinate equal to 2^D, which the table does
//   not cover, walk from the root.
#pragma once
#include "ve_device.cuh"

namespace ve {
namespace dev {

struct RayCount {
    uint32_t fetch = 0;
    uint32_t steps = 0;
};

__device__ __forceinline__ uint32_t fetch_node(const uint32_t* __restrict__ nodes, uint64_t n, uint32_t off) {
    return off < n ? __ldg(nodes + off) : 0u;
}


// The bound of a node array as the trace kernel keeps it: offsets are 32-bit,
// so a bound clamped to 2^32 - 1 rejects exactly the same offsets.
__device__ __forceinline__ uint32_t word_bound(uint64_t n) { return n < 0xFFFFFFFFull ? uint32_t(n) : 0xFFFFFFFFu; }
// The DDA as a resumable state machine: dda_init performs the origin advance
// and the entry intersection, dda_step one iteration of the reference loop
// `while (inBounds(r_pos) && q++ <= controlchecks)`.  Both return true when
// the ray is finished, with the result in `h`.
struct Dda {
    f3 o, d, inv;
    float t;  // the position is d * t + o (recomputed each step: the same operations as storing it)
    float t_end;  // CLIP: past this distance the ray can hit nothing (set by the caller)
    uint32_t q, cc;
    uint32_t lux, luy, luz, e_last;
    uint32_t bD;  // FLAT: offset of the leaf block (the child block reached at level D)
    uint32_t base[17];
};

__device__ __forceinline__ bool dda_init(Dda& s, f3 o, f3 d, uint32_t controlchecks, uint32_t D, Hit& h) {
    const float Lf = float(1u << D);
    h.status = kEscaped;
    h.id = 0;
    h.material = 0;
    h.x = h.y = h.z = 0;
    h.size = 0;
    s.inv = mk(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
    s.d = d;
    s.o = add(o, muls(d, 4.0f));
    s.q = 0;
    s.cc = controlchecks;
    s.base[0] = 0u;
    // no position yet: every bit differs from the first step's, which
    // therefore restarts at level 0
    s.lux = s.luy = s.luz = 0xFFFFFFFFu;
    s.e_last = 0;
    if (in_bounds(s.o, Lf)) {
        s.t = 0.0f;
    } else {
        const f3 t1 = mul(mk((0.0f - s.o.x) + 0.001f, (0.0f - s.o.y) + 0.001f, (0.0f - s.o.z) + 0.001f), s.inv);
        const f3 t2 = mul(mk((Lf - s.o.x) - 0.001f, (Lf - s.o.y) - 0.001f, (Lf - s.o.z) - 0.001f), s.inv);
        const float t_enter = gmax(gmax(gmin(t1.x, t2.x), gmin(t1.y, t2.y)), gmin(t1.z, t2.z));
        const float t_exit = gmin(gmin(gmax(t1.x, t2.x), gmax(t1.y, t2.y)), gmax(t1.z, t2.z));
        s.q++;
        if (t_exit < t_enter || t_exit < 0.0f) {
            h.checks = s.q;
            return true;
        }
        s.t = t_enter;
    }
    return false;
}

// Top-table entry of the cell containing (x, y, z): (offset << 1) | 1 when
// levels 0..T0-1 are internal (offset = child block of the level-T0 node),
// else (terminal level << 1).  The table covers positions below 2^D on every
// axis (root child 0, which level 0's bit-D test selects for them).
__device__ __forceinline__ uint32_t top_index(uint32_t x, uint32_t y, uint32_t z, uint32_t D, uint32_t T0) {
    const uint32_t sh = D - T0 + 1u, b = T0 - 1u;
    return ((((x >> sh) << b) | (y >> sh)) << b) | (z >> sh);
}

// WORD: a hit reports the leaf's node word in h.id instead of its slot (the
// bounce trace keeps the word for shading; the slot is the GBuffer's field).
// CLIP: the ray also ends, as escaped, once its distance passes s.t_end —
// for callers to whom an escape and a timeout are the same result.
// FLAT: the scene's top table reaches the leaves (T0 = D): a descent is one
// table word, then the leaf word, and the only offset kept across steps is
// the leaf block's (a register, not the per-level array).
template <bool COUNT, bool WORD = false, bool CLIP = false, bool FLAT = false>
__device__ __forceinline__ bool dda_step(Dda& s, const uint32_t* __restrict__ nodes, uint64_t n_words, uint32_t D,
                                         const uint32_t* __restrict__ top, uint32_t T0, Hit& h, RayCount& rc) {
    const uint32_t L = 1u << D;
    const float Lf = float(L);
    const f3 r = add(muls(s.d, s.t), s.o);
    if (!in_bounds(r, Lf) || (CLIP && s.t > s.t_end)) {
        h.status = kEscaped;
        h.checks = s.q;
        return true;
    }
    if (!(s.q++ <= s.cc)) {
        h.status = kTimeout;
        h.checks = s.q;
        return true;
    }
    if (COUNT) rc.steps++;
    const uint32_t ux = uint32_t(r.x), uy = uint32_t(r.y), uz = uint32_t(r.z);
    bool reuse = false;
    uint32_t start = 0;
    {
        const uint32_t xd = (ux ^ s.lux) | (uy ^ s.luy) | (uz ^ s.luz);
        if (xd == 0u) {
            reuse = true;
        } else {
            const uint32_t hb = 31u - uint32_t(__clz(xd));
            start = hb >= D ? 0u : D - hb;
            reuse = start > s.e_last;
        }
    }
    uint32_t k = s.e_last;
    if (FLAT && !reuse) {
        s.lux = ux; s.luy = uy; s.luz = uz;
        bool found = false;
        k = start;
        const uint32_t sx = ux << 2, sy = uy << 1;
        if (start < D) {
            if (!((ux | uy | uz) & L)) {
                const uint32_t ent = __ldg(top + top_index(ux, uy, uz, D, T0));
                if (ent & 1u) {
                    s.bD = ent >> 1;
                    k = D;
                } else {
                    k = ent >> 1;
                    found = true;
                }
            } else {
                // a coordinate equal to 2^D (outside the table's cells): the
                // walk from the root, reading the words the restart would
                uint32_t b = 0u;
                for (k = 0; k < D; k++) {
                    const uint32_t sh = D - k;
                    const uint32_t raw = fetch_node(nodes, n_words,
                                                    b + (((sx >> sh) & 4u) | ((sy >> sh) & 2u) | ((uz >> sh) & 1u)));
                    if (!(raw & 1u)) {
                        found = true;
                        break;
                    }
                    b = raw >> 4;
                }
                if (!found) s.bD = b;
            }
        }
        s.e_last = k;
        if (!found) {
            const uint32_t off = s.bD + ((sx & 4u) | (sy & 2u) | (uz & 1u));
            const uint32_t raw = fetch_node(nodes, n_words, off);
            const uint32_t mat = (raw & 254u) >> 1;
            if (mat != 0u) {
                h.status = kHit;
                h.id = WORD ? raw : off;
                h.material = mat;
                h.x = ux; h.y = uy; h.z = uz;
                h.size = 1u;
                h.checks = s.q;
                return true;
            }
        }
    } else if (!reuse) {
        s.lux = ux; s.luy = uy; s.luz = uz;
        bool found = false;
        uint32_t off = 0;
        k = start;
        // child index at level k: bit D-k of x, y, z as bits 2, 1, 0
        const uint32_t sx = ux << 2, sy = uy << 1;
        // inBounds admits a coordinate equal to 2^D; level 0 then selects
        // another root child than the table's, so such a position walks
        // every level as the reference's descent does
        if (!COUNT && start < T0 && !((ux | uy | uz) & L)) {
            const uint32_t ent = __ldg(top + top_index(ux, uy, uz, D, T0));
            if (ent & 1u) {
                s.base[T0] = ent >> 1;
                k = T0;
            } else {
                k = ent >> 1;
                found = true;
            }
        }
        for (; !found && k < D; k++) {
            const uint32_t b = D - k;  // the position bit level k tests
            off = s.base[k] + (((sx >> b) & 4u) | ((sy >> b) & 2u) | ((uz >> b) & 1u));
            const uint32_t raw = fetch_node(nodes, n_words, off);
            if (COUNT) rc.fetch++;
            if (!(raw & 1u)) {
                found = true;
                break;
            }
            s.base[k + 1] = raw >> 4;
        }
        s.e_last = k;
        if (!found) {
            off = s.base[D] + ((sx & 4u) | (sy & 2u) | (uz & 1u));
            const uint32_t raw = fetch_node(nodes, n_words, off);
            if (COUNT) rc.fetch++;
            const uint32_t mat = (raw & 254u) >> 1;
            if (mat != 0u) {
                h.status = kHit;
                h.id = WORD ? raw : off;
                h.material = mat;
                h.x = ux; h.y = uy; h.z = uz;
                h.size = 1u;
                h.checks = s.q;
                return true;
            }
        }
    }
    const uint32_t size = L >> k;
    const uint32_t px = ux & ~(size - 1u), py = uy & ~(size - 1u), pz = uz & ~(size - 1u);
    // exit of the cell: the reference takes, per axis, the larger of the two
    // slab distances ((min - o) - 0.001) / d and ((max - o) + 0.001) / d.
    // Rounding is monotone and the first numerator is below the second, so
    // that larger one is always the second where 1/d > 0 (+inf included) and
    // the first elsewhere: only that plane is computed, with the same
    // operations, giving the same bits (3-4 % less trace time than both).
    const bool ax = s.inv.x > 0.0f, ay = s.inv.y > 0.0f, az = s.inv.z > 0.0f;
    const float tx = ((float(px + (ax ? size : 0u)) - s.o.x) + (ax ? 0.001f : -0.001f)) * s.inv.x;
    const float ty = ((float(py + (ay ? size : 0u)) - s.o.y) + (ay ? 0.001f : -0.001f)) * s.inv.y;
    const float tz = ((float(pz + (az ? size : 0u)) - s.o.z) + (az ? 0.001f : -0.001f)) * s.inv.z;
    const float t_exit = gmin(gmin(tx, ty), tz);
    s.t = t_exit;
    return false;
}

template <bool COUNT>
__device__ __forceinline__ Hit raycast(const uint32_t* __restrict__ nodes, uint64_t n_words, uint32_t D,
                                       const uint32_t* __restrict__ top, uint32_t T0, f3 o, f3 d,
                                       uint32_t controlchecks, RayCount& rc) {
    Dda s;
    Hit h;
    if (dda_init(s, o, d, controlchecks, D, h)) return h;
    if (!COUNT && T0 == D) {
        while (!dda_step<COUNT, false, false, true>(s, nodes, n_words, D, top, T0, h, rc)) {
        }
    } else {
        while (!dda_step<COUNT>(s, nodes, n_words, D, top, T0, h, rc)) {
        }
    }
    return h;
}

}  // namespace dev
}  // namespace ve
