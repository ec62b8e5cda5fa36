// terrain_oracle.cpp — TEST INFRASTRUCTURE ONLY: the benchmark scenes for the
// CPU side (the oracle and the timed reference arm), built without the
// product library.
//
// The scene is the seeded value-noise terrain of the benchmark workloads:
// column heights 64 + 32·fBm2(x/32, z/32) (4 octaves, gain 0.5, lacunarity 2),
// solid below the height; variant 1 adds a ±16-voxel band in which 3 octaves of
// 3D value noise carve overhangs; variant 2 is variant 1 restricted to the
// central 1024² columns.  Materials are 1 + hash(x, y, z) mod 8.
//
// The node words follow Octree::set (src/renderer/octree.cpp:127-217):
// slot 0 = root {isNode, count, next = 1}, slots 1-8 = the root's children,
// every internal node an 8-slot block at `size` (from 9, step 8) in the order
// of set's iterative DFS — the root's children processed 0..7, each subtree's
// children pushed 0..7 and popped 7..0, i.e. a pre-order walk visiting
// children 7..0 (octree.cpp:203-214) — leaves {isNode = 0, material & 0x7F}
// (:192-196), empty children 0.  Instead of a pointer tree (≈100 B per node,
// too large at depth 10) it walks an occupancy pyramid: one bit per cell of
// every level.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace {

inline uint32_t mix32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

inline uint32_t seed32(uint64_t seed, uint32_t salt) {
    return mix32(uint32_t(seed) ^ mix32(uint32_t(seed >> 32) ^ salt));
}

// lattice value in [-1, 1) of integer point (ix, iy, iz) under salt s
inline double lattice(int64_t ix, int64_t iy, int64_t iz, uint32_t s) {
    const uint32_t hz = mix32(uint32_t(iz) * 0xcb1ab31fu ^ s);
    const uint32_t hy = mix32(uint32_t(iy) * 0xd8163841u ^ hz);
    const uint32_t h = mix32(uint32_t(ix) * 0x8da6b343u ^ hy);
    return double(h >> 8) * (2.0 / 16777216.0) - 1.0;
}

inline double smooth(double t) { return t * t * (3.0 - 2.0 * t); }
inline double lerp(double a, double b, double t) { return a + (b - a) * t; }

double value2(double x, double z, uint32_t s) {
    const double fx = std::floor(x), fz = std::floor(z);
    const int64_t ix = int64_t(fx), iz = int64_t(fz);
    const double u = smooth(x - fx), v = smooth(z - fz);
    const double row0 = lerp(lattice(ix, 0, iz, s), lattice(ix + 1, 0, iz, s), u);
    const double row1 = lerp(lattice(ix, 0, iz + 1, s), lattice(ix + 1, 0, iz + 1, s), u);
    return row0 + (row1 - row0) * v;
}

double value3(double x, double y, double z, uint32_t s) {
    const double fx = std::floor(x), fy = std::floor(y), fz = std::floor(z);
    const int64_t ix = int64_t(fx), iy = int64_t(fy), iz = int64_t(fz);
    const double u = smooth(x - fx), v = smooth(y - fy), w = smooth(z - fz);
    const double a00 = lerp(lattice(ix, iy, iz, s), lattice(ix + 1, iy, iz, s), u);
    const double a10 = lerp(lattice(ix, iy + 1, iz, s), lattice(ix + 1, iy + 1, iz, s), u);
    const double a01 = lerp(lattice(ix, iy, iz + 1, s), lattice(ix + 1, iy, iz + 1, s), u);
    const double a11 = lerp(lattice(ix, iy + 1, iz + 1, s), lattice(ix + 1, iy + 1, iz + 1, s), u);
    return lerp(lerp(a00, a10, v), lerp(a01, a11, v), w);
}

double fbm(int dims, double x, double y, double z, int octaves, uint32_t s) {
    double sum = 0.0, amp = 1.0, freq = 1.0, norm = 0.0;
    for (int o = 0; o < octaves; o++) {
        const uint32_t so = s + uint32_t(o) * 0x9E3779B9u;
        sum += amp * (dims == 2 ? value2(x * freq, z * freq, so) : value3(x * freq, y * freq, z * freq, so));
        norm += amp;
        amp *= 0.5;
        freq *= 2.0;
    }
    return sum / norm;
}

template <typename F>
void parallel_rows(uint32_t n, uint32_t threads, F&& fn) {
    threads = std::max(1u, std::min(threads, n));
    std::atomic<uint32_t> next{0};
    std::vector<std::thread> th;
    for (uint32_t t = 0; t < threads; t++)
        th.emplace_back([&] {
            for (uint32_t i; (i = next.fetch_add(1)) < n;) fn(i);
        });
    for (auto& t : th) t.join();
}

struct Scene {
    uint32_t D, L, variant;
    uint64_t seed;
    float band;
    std::vector<float> height;                 // [z * L + x]
    std::vector<std::vector<uint64_t>> occ;   // level k: one bit per cell, index (x * n + y) * n + z

    bool solid(uint32_t x, uint32_t y, uint32_t z) const {
        const double yc = double(y) + 0.5;
        const double h = double(height[size_t(z) * L + x]);
        if (variant == 0) return yc < h;
        const double A = band;
        if (yc < h - A) return true;
        if (yc >= h + A) return false;
        const double f = fbm(3, (x + 0.5) / 24.0, yc / 24.0, (z + 0.5) / 24.0, 3, seed32(seed, 0x4f56u));
        return yc < h + A * f;
    }
    uint32_t material(uint32_t x, uint32_t y, uint32_t z) const {
        const uint32_t s = seed32(seed, 0x4d41u);
        return 1u + mix32(x * 0x9E3779B1u ^ mix32(y * 0x85EBCA77u ^ mix32(z * 0xC2B2AE3Du ^ s))) % 8u;
    }
    bool occupied(uint32_t k, uint32_t x, uint32_t y, uint32_t z) const {
        const uint64_t n = 1ull << k;
        const uint64_t i = (uint64_t(x) * n + y) * n + z;
        return (occ[k][i >> 6] >> (i & 63)) & 1u;
    }
};

void make_scene(Scene& S, uint32_t depth, uint32_t variant, uint64_t seed, uint32_t threads) {
    S.D = depth;
    S.L = 1u << depth;
    S.variant = variant;
    S.seed = seed;
    S.band = variant != 0 ? 16.0f : 0.0f;
    const uint32_t L = S.L;
    S.height.assign(size_t(L) * L, 0.0f);
    const uint32_t sh = seed32(seed, 0x4845u);
    parallel_rows(L, threads, [&](uint32_t z) {
        for (uint32_t x = 0; x < L; x++)
            S.height[size_t(z) * L + x] = float(64.0 + 32.0 * fbm(2, (x + 0.5) / 32.0, 0.0, (z + 0.5) / 32.0, 4, sh));
    });
    if (variant == 2 && L > 1024u) {
        const uint32_t lo = (L - 1024u) / 2u;
        for (uint32_t z = 0; z < L; z++)
            for (uint32_t x = 0; x < L; x++)
                if (x < lo || z < lo || x >= lo + 1024u || z >= lo + 1024u) S.height[size_t(z) * L + x] = -1.0e6f;
    }
    S.occ.resize(depth + 1);
    for (uint32_t k = 0; k <= depth; k++) {
        const uint64_t cells = 1ull << (3 * k);
        S.occ[k].assign((cells + 63) / 64, 0ull);
    }
    // leaf level: x-major rows of 64 z-bits (a y-column of one x is L² bits)
    double top = 0.0;
    for (float h : S.height) top = std::max(top, double(h));
    const uint32_t ymax = uint32_t(std::min<double>(L, std::max(0.0, std::ceil(top + S.band)) + 1.0));
    std::vector<uint64_t>& leaf = S.occ[depth];
    // one x per task: tasks share no 64-bit word once a plane holds >= 64 cells
    parallel_rows(L, L >= 8 ? threads : 1u, [&](uint32_t x) {
        for (uint32_t y = 0; y < ymax; y++)
            for (uint32_t z = 0; z < L; z++)
                if (S.solid(x, y, z)) {
                    const uint64_t i = (uint64_t(x) * L + y) * L + z;
                    leaf[i >> 6] |= 1ull << (i & 63);
                }
    });
    for (int k = int(depth) - 1; k >= 0; k--) {
        const uint32_t n = 1u << k;
        parallel_rows(n, n >= 8 ? threads : 1u, [&](uint32_t x) {
            for (uint32_t y = 0; y < n; y++)
                for (uint32_t z = 0; z < n; z++) {
                    bool any = false;
                    for (uint32_t c = 0; c < 8 && !any; c++)
                        any = S.occupied(uint32_t(k) + 1, 2 * x + ((c >> 2) & 1), 2 * y + ((c >> 1) & 1), 2 * z + (c & 1));
                    if (any) {
                        const uint64_t i = (uint64_t(x) * n + y) * n + z;
                        S.occ[k][i >> 6] |= 1ull << (i & 63);
                    }
                }
        });
    }
}

struct Emit {
    const Scene& S;
    std::vector<uint32_t>& data;
    uint64_t size = 9;
    uint64_t voxels = 0;
    bool overflow = false;

    uint32_t child_count(uint32_t k, uint32_t x, uint32_t y, uint32_t z) const {
        uint32_t c = 0;
        for (uint32_t i = 0; i < 8; i++)
            c += S.occupied(k + 1, 2 * x + ((i >> 2) & 1), 2 * y + ((i >> 1) & 1), 2 * z + (i & 1));
        return c;
    }
    // an occupied cell at level k (1 <= k <= D) written into `slot`
    void node(uint32_t k, uint32_t x, uint32_t y, uint32_t z, uint64_t slot) {
        if (k == S.D) {
            data[slot] = (S.material(x, y, z) & 0x7Fu) << 1;
            voxels++;
            return;
        }
        const uint64_t block = size;
        size += 8;
        if (size > (1ull << 28)) overflow = true;
        if (data.size() < size) data.resize(std::max<uint64_t>(size, data.size() * 3 / 2), 0u);
        data[slot] = 1u | ((child_count(k, x, y, z) & 7u) << 1) | (uint32_t(block) << 4);
        for (int i = 7; i >= 0; i--) {
            const uint32_t cx = 2 * x + ((i >> 2) & 1), cy = 2 * y + ((i >> 1) & 1), cz = 2 * z + (i & 1);
            if (S.occupied(k + 1, cx, cy, cz)) node(k + 1, cx, cy, cz, block + uint64_t(i));
        }
    }
};

struct TerrainWords {
    std::vector<uint32_t> data;
    uint64_t voxels = 0;
};

}  // namespace

extern "C" {

// Builds the node words of the terrain scene (depth >= 1); returns a handle
// (null when the tree does not fit the 28-bit `next` field) with the word and
// leaf counts in *n_words and *n_voxels.  Read the words with
// oracle_terrain_data, release with oracle_terrain_free.
void* oracle_terrain_build(uint32_t depth, uint32_t variant, uint64_t seed, uint32_t threads, uint64_t* n_words,
                           uint64_t* n_voxels) {
    if (threads == 0) threads = std::max(1u, std::thread::hardware_concurrency());
    *n_words = 0;
    *n_voxels = 0;
    if (depth < 1 || depth > 11) return nullptr;
    Scene S;
    make_scene(S, depth, variant, seed, threads);
    auto* t = new TerrainWords;
    t->data.assign(9, 0u);
    if (S.occupied(0, 0, 0, 0)) {  // else Octree::set on an empty OctreeCPU: 9 zero words
        Emit e{S, t->data};
        uint32_t root_count = 0;
        for (uint32_t c = 0; c < 8; c++) root_count += S.occupied(1, (c >> 2) & 1, (c >> 1) & 1, c & 1);
        t->data[0] = 1u | ((root_count & 7u) << 1) | (1u << 4);
        for (uint32_t c = 0; c < 8; c++) {
            const uint32_t x = (c >> 2) & 1, y = (c >> 1) & 1, z = c & 1;
            if (S.occupied(1, x, y, z)) e.node(1, x, y, z, 1 + c);
        }
        if (e.overflow) {
            delete t;
            return nullptr;
        }
        t->data.resize(e.size);
        t->voxels = e.voxels;
    }
    *n_words = t->data.size();
    *n_voxels = t->voxels;
    return t;
}

const uint32_t* oracle_terrain_data(const void* h) { return static_cast<const TerrainWords*>(h)->data.data(); }

void oracle_terrain_free(void* h) { delete static_cast<TerrainWords*>(h); }
// The benchmark material table: 128 std140 Material entries of 16 floats;
// materials 1-8 get albedo U[0.2, 0.9]^3 from a splitmix64 stream, roughness 1,
// no specular, no metal, no emission.
void oracle_terrain_materials(uint64_t seed, float out[128 * 16]) {
    std::memset(out, 0, sizeof(float) * 128 * 16);
    uint64_t s = seed ^ 0x6d6174657269616cull;
    auto next = [&s]() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    };
    for (int i = 1; i <= 8; i++) {
        float* m = out + 16 * i;
        for (int c = 0; c < 3; c++) {
            const double u = double(next() >> 11) * (1.0 / 9007199254740992.0);
            m[c] = float(0.2 + 0.7 * u);  // color
            m[4 + c] = m[c];              // specularColor
        }
        m[3] = 0.0f;
        m[7] = 1.0f;
        m[8] = 1.0f;  // roughness
    }
}

}  // extern "C"
