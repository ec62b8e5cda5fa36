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

template <bool COUNT>
__device__ __forceinline__ Hit raycast(const uint32_t* __restrict__ nodes, uint64_t n_words, uint32_t D, f3 o, f3 d,
                                       uint32_t controlchecks, RayCount& rc) {
    const uint32_t L = 1u << D;
    const float Lf = float(L);
    Hit h;
    h.status = kEscaped;
    h.id = 0;
    h.material = 0;
    h.x = h.y = h.z = 0;
    h.size = 0;
    const f3 inv = mk(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
    o = add(o, muls(d, 4.0f));
    uint32_t q = 0;
    f3 r;
    if (in_bounds(o, Lf)) {
        r = o;
    } else {
        const f3 t1 = mul(mk((0.0f - o.x) + 0.001f, (0.0f - o.y) + 0.001f, (0.0f - o.z) + 0.001f), inv);
        const f3 t2 = mul(mk((Lf - o.x) - 0.001f, (Lf - o.y) - 0.001f, (Lf - o.z) - 0.001f), inv);
        const float t_enter = gmax(gmax(gmin(t1.x, t2.x), gmin(t1.y, t2.y)), gmin(t1.z, t2.z));
        const float t_exit = gmin(gmin(gmax(t1.x, t2.x), gmax(t1.y, t2.y)), gmax(t1.z, t2.z));
        q++;
        if (t_exit < t_enter || t_exit < 0.0f) {
            h.checks = q;
            return h;
        }
        r = add(muls(d, t_enter), o);
    }
    uint32_t base[17];
    base[0] = 0u;
    uint32_t lux = 0, luy = 0, luz = 0, e_last = 0;
    bool first = true;
    while (in_bounds(r, Lf) && q++ <= controlchecks) {
        if (COUNT) rc.steps++;
        const uint32_t ux = uint32_t(r.x), uy = uint32_t(r.y), uz = uint32_t(r.z);
        bool reuse = false;
        uint32_t start = 0;
        if (!first) {
            const uint32_t xd = (ux ^ lux) | (uy ^ luy) | (uz ^ luz);
            if (xd == 0u) {
                reuse = true;
            } else {
                const uint32_t hb = 31u - uint32_t(__clz(xd));
                start = hb >= D ? 0u : D - hb;
                reuse = start > e_last;
            }
        }
        uint32_t k = e_last;
        if (!reuse) {
            first = false;
            lux = ux; luy = uy; luz = uz;
            bool found = false;
            uint32_t off = 0;
            for (k = start; k < D; k++) {
                off = base[k] + locate(ux, uy, uz, L >> k);
                const uint32_t raw = fetch_node(nodes, n_words, off);
                if (COUNT) rc.fetch++;
                if (!(raw & 1u)) {
                    found = true;
                    break;
                }
                base[k + 1] = raw >> 4;
            }
            e_last = k;
            if (!found) {
                off = base[D] + locate(ux, uy, uz, 1u);
                const uint32_t raw = fetch_node(nodes, n_words, off);
                if (COUNT) rc.fetch++;
                const uint32_t mat = (raw & 254u) >> 1;
                if (mat != 0u) {
                    h.status = kHit;
                    h.id = off;
                    h.material = mat;
                    h.x = ux; h.y = uy; h.z = uz;
                    h.size = 1u;
                    h.checks = q;
                    return h;
                }
            }
        }
        const uint32_t size = L >> k;
        const uint32_t px = ux & ~(size - 1u), py = uy & ~(size - 1u), pz = uz & ~(size - 1u);
        const f3 bmin = mk(float(px), float(py), float(pz));
        const float fs = float(size);
        const f3 t1 = mul(mk((bmin.x - o.x) - 0.001f, (bmin.y - o.y) - 0.001f, (bmin.z - o.z) - 0.001f), inv);
        const f3 t2 = mul(mk(((bmin.x + fs) - o.x) + 0.001f, ((bmin.y + fs) - o.y) + 0.001f,
                             ((bmin.z + fs) - o.z) + 0.001f),
                          inv);
        const float t_exit = gmin(gmin(gmax(t1.x, t2.x), gmax(t1.y, t2.y)), gmax(t1.z, t2.z));
        r = add(muls(d, t_exit), o);
    }
    h.status = in_bounds(r, Lf) ? kTimeout : kEscaped;
    h.checks = q;
    return h;
}

}  // namespace dev
}  // namespace ve
