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
// The walk is a per-lane state machine: one dda_iter call performs at most
// one exit computation (leave the terminal cell, loop test, restart level)
// and one node fetch, so lanes whose descents differ in depth stay in step
// instead of the whole warp waiting for its deepest descent.
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

// 8-bit mask of the leaf words (material != 0) of the block starting at slot
// `b`.  Blocks of the reference layout start at slots 1 + 8k, which the
// device array's 7-word offset puts on 32-byte boundaries: two 128-bit loads.
__device__ __forceinline__ uint32_t leaf_block_mask(const uint32_t* __restrict__ nodes, uint64_t n, uint32_t b) {
    uint32_t w[8];
    if ((b & 7u) == 1u && uint64_t(b) + 8u <= n) {
        const uint4 lo = __ldg(reinterpret_cast<const uint4*>(nodes + b));
        const uint4 hi = __ldg(reinterpret_cast<const uint4*>(nodes + b + 4));
        w[0] = lo.x; w[1] = lo.y; w[2] = lo.z; w[3] = lo.w;
        w[4] = hi.x; w[5] = hi.y; w[6] = hi.z; w[7] = hi.w;
    } else {
#pragma unroll
        for (int i = 0; i < 8; i++) w[i] = fetch_node(nodes, n, b + uint32_t(i));
    }
    uint32_t m = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) m |= uint32_t((w[i] & 254u) != 0u) << i;
    return m;
}

// Scalar DDA state (registers); the descent stack `base` (child-block offset
// per level, dynamically indexed) is a separate local array.
struct Dda {
    f3 o, d, inv, r;
    uint32_t q, cc;
    uint32_t ux, uy, uz;            // integer position of the current step
    uint32_t e_last;                // terminal level of the current step's cell
    uint32_t k;                     // next level to fetch while descending
    uint32_t leaf_base, leaf_mask;  // leaf-level block cached as an 8-bit "has material" mask
    bool descending;
};

// Loop test of the reference (`inBounds(r_pos) && q++ <= controlchecks`) for
// the position s.r; on failure the ray ends (escaped / out of checks).
__device__ __forceinline__ bool dda_loop_test(Dda& s, float Lf, Hit& h) {
    if (!in_bounds(s.r, Lf)) {
        h.status = kEscaped;
        h.checks = s.q;
        return false;
    }
    if (!(s.q++ <= s.cc)) {
        h.status = kTimeout;
        h.checks = s.q;
        return false;
    }
    return true;
}

// Origin advance, entry intersection (intersect, internal.glsl:245-253) and
// the first loop test.  Returns true when the ray is already finished.
template <bool COUNT>
__device__ __forceinline__ bool dda_init(Dda& s, uint32_t* base, f3 o, f3 d, uint32_t controlchecks, uint32_t D,
                                         Hit& h, RayCount& rc) {
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
    base[0] = 0u;
    s.e_last = 0;
    s.leaf_base = 0xFFFFFFFFu;
    s.leaf_mask = 0u;
    if (in_bounds(s.o, Lf)) {
        s.r = s.o;
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
        s.r = add(muls(d, t_enter), s.o);
    }
    if (!dda_loop_test(s, Lf, h)) return true;
    if (COUNT) rc.steps++;
    s.ux = uint32_t(s.r.x);
    s.uy = uint32_t(s.r.y);
    s.uz = uint32_t(s.r.z);
    s.descending = true;
    s.k = 0;
    return false;
}

// One iteration: (a) when the current cell is known, leave it
// (intersect_inside, internal.glsl:255-261), run the loop test and pick the
// restart level for the new position; (b) when descending, read one node.
// Returns true when the ray is finished (hit, escaped or out of checks).
template <bool COUNT>
__device__ __forceinline__ bool dda_iter(Dda& s, uint32_t* base, const uint32_t* __restrict__ nodes,
                                         uint64_t n_words, uint32_t D, Hit& h, RayCount& rc) {
    const uint32_t L = 1u << D;
    if (!s.descending) {
        const uint32_t size = L >> s.e_last;
        const f3 bmin = mk(float(s.ux & ~(size - 1u)), float(s.uy & ~(size - 1u)), float(s.uz & ~(size - 1u)));
        const float fs = float(size);
        const f3 t1 = mul(mk((bmin.x - s.o.x) - 0.001f, (bmin.y - s.o.y) - 0.001f, (bmin.z - s.o.z) - 0.001f), s.inv);
        const f3 t2 = mul(mk(((bmin.x + fs) - s.o.x) + 0.001f, ((bmin.y + fs) - s.o.y) + 0.001f,
                             ((bmin.z + fs) - s.o.z) + 0.001f),
                          s.inv);
        const float t_exit = gmin(gmin(gmax(t1.x, t2.x), gmax(t1.y, t2.y)), gmax(t1.z, t2.z));
        s.r = add(muls(s.d, t_exit), s.o);
        if (!dda_loop_test(s, float(L), h)) return true;
        if (COUNT) rc.steps++;
        const uint32_t nx = uint32_t(s.r.x), ny = uint32_t(s.r.y), nz = uint32_t(s.r.z);
        const uint32_t xd = (nx ^ s.ux) | (ny ^ s.uy) | (nz ^ s.uz);
        s.ux = nx; s.uy = ny; s.uz = nz;
        if (xd != 0u) {
            const uint32_t hb = 31u - uint32_t(__clz(xd));
            const uint32_t start = hb >= D ? 0u : D - hb;
            if (start <= s.e_last) {  // the new position leaves the terminal cell: descend from `start`
                s.descending = true;
                s.k = start;
            }
        }
        // otherwise the position is still inside the same terminal cell
    }
    if (s.descending) {
        if (s.k < D) {
            const uint32_t off = base[s.k] + locate(s.ux, s.uy, s.uz, L >> s.k);
            const uint32_t raw = fetch_node(nodes, n_words, off);
            if (COUNT) rc.fetch++;
            if (!(raw & 1u)) {  // empty or compressed: terminal cell, never a hit
                s.e_last = s.k;
                s.descending = false;
            } else {
                base[s.k + 1] = raw >> 4;
                s.k++;
            }
        } else {
            const uint32_t lb = base[D];
            if (lb != s.leaf_base) {
                s.leaf_base = lb;
                s.leaf_mask = leaf_block_mask(nodes, n_words, lb);
            }
            const uint32_t li = locate(s.ux, s.uy, s.uz, 1u);
            if (COUNT) rc.fetch++;
            if ((s.leaf_mask >> li) & 1u) {
                const uint32_t off = lb + li;
                h.status = kHit;
                h.id = off;
                h.material = (fetch_node(nodes, n_words, off) & 254u) >> 1;
                h.x = s.ux; h.y = s.uy; h.z = s.uz;
                h.size = 1u;
                h.checks = s.q;
                return true;
            }
            s.e_last = D;
            s.descending = false;
        }
    }
    return false;
}

template <bool COUNT>
__device__ __forceinline__ Hit raycast(const uint32_t* __restrict__ nodes, uint64_t n_words, uint32_t D, f3 o, f3 d,
                                       uint32_t controlchecks, RayCount& rc) {
    Dda s;
    uint32_t base[17];
    Hit h;
    if (dda_init<COUNT>(s, base, o, d, controlchecks, D, h, rc)) return h;
    while (!dda_iter<COUNT>(s, base, nodes, n_words, D, h, rc)) {
    }
    return h;
}

}  // namespace dev
}  // namespace ve
