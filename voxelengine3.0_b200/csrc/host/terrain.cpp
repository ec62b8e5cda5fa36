// terrain.cpp — seeded value-noise terrain scenes, their parallel bulk
// octree builder, the camera basis and the benchmark material table.
//
// The bulk builder emits exactly the words OctreeCPU::insert followed by
// Octree::set would produce (src/renderer/octree.cpp:127-217): slot 0 root
// {next = 1}, slots 1-8 the root's children, and one 8-slot block per
// internal node allocated in DFS pre-order — root children in order 0..7,
// every other node's children in order 7..0 (the LIFO pop order of
// linearizeNode).  It works on an occupancy pyramid instead of pointer nodes:
//   1. 8^3-voxel bricks: a 512-bit occupancy mask per brick (parallel);
//   2. per brick the occupied 4^3 and 2^3 sub-cubes; above bricks a byte
//      pyramid of occupied cells;
//   3. internal-node counts per level-2 subtree give every subtree's first
//      block, so the 64 level-2 subtrees are emitted in parallel.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <thread>

#include "scene_host.h"

namespace ve {

namespace {

inline uint32_t mix32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
inline uint64_t splitmix64(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
inline double lattice(int64_t ix, int64_t iy, int64_t iz, uint32_t s) {
    uint32_t h = mix32(uint32_t(ix) * 0x8da6b343u ^ mix32(uint32_t(iy) * 0xd8163841u ^ mix32(uint32_t(iz) * 0xcb1ab31fu ^ s)));
    return double(h >> 8) * (2.0 / 16777216.0) - 1.0;
}
inline double fade(double t) { return t * t * (3.0 - 2.0 * t); }
double noise2(double x, double z, uint32_t s) {
    const double fx0 = std::floor(x), fz0 = std::floor(z);
    const int64_t x0 = int64_t(fx0), z0 = int64_t(fz0);
    const double u = fade(x - fx0), v = fade(z - fz0);
    const double a = lattice(x0, 0, z0, s), b = lattice(x0 + 1, 0, z0, s);
    const double c = lattice(x0, 0, z0 + 1, s), d = lattice(x0 + 1, 0, z0 + 1, s);
    return (a + (b - a) * u) + ((c + (d - c) * u) - (a + (b - a) * u)) * v;
}
double noise3(double x, double y, double z, uint32_t s) {
    const double fx0 = std::floor(x), fy0 = std::floor(y), fz0 = std::floor(z);
    const int64_t x0 = int64_t(fx0), y0 = int64_t(fy0), z0 = int64_t(fz0);
    const double u = fade(x - fx0), v = fade(y - fy0), w = fade(z - fz0);
    double c[2][2][2];
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++)
            for (int k = 0; k < 2; k++) c[i][j][k] = lattice(x0 + i, y0 + j, z0 + k, s);
    auto lerp = [](double a, double b, double t) { return a + (b - a) * t; };
    const double x00 = lerp(c[0][0][0], c[1][0][0], u), x10 = lerp(c[0][1][0], c[1][1][0], u);
    const double x01 = lerp(c[0][0][1], c[1][0][1], u), x11 = lerp(c[0][1][1], c[1][1][1], u);
    return lerp(lerp(x00, x10, v), lerp(x01, x11, v), w);
}
double fbm2(double x, double z, int octaves, uint32_t s) {
    double sum = 0, amp = 1, freq = 1, norm = 0;
    for (int o = 0; o < octaves; o++) {
        sum += amp * noise2(x * freq, z * freq, s + uint32_t(o) * 0x9E3779B9u);
        norm += amp;
        amp *= 0.5;
        freq *= 2.0;
    }
    return sum / norm;
}
double fbm3(double x, double y, double z, int octaves, uint32_t s) {
    double sum = 0, amp = 1, freq = 1, norm = 0;
    for (int o = 0; o < octaves; o++) {
        sum += amp * noise3(x * freq, y * freq, z * freq, s + uint32_t(o) * 0x9E3779B9u);
        norm += amp;
        amp *= 0.5;
        freq *= 2.0;
    }
    return sum / norm;
}
inline uint32_t seed32(uint64_t seed, uint32_t salt) {
    return mix32(uint32_t(seed) ^ mix32(uint32_t(seed >> 32) ^ salt));
}

void parallel_for(uint32_t n, uint32_t threads, const std::function<void(uint32_t)>& fn) {
    if (threads <= 1 || n <= 1) {
        for (uint32_t i = 0; i < n; i++) fn(i);
        return;
    }
    std::atomic<uint32_t> next{0};
    std::vector<std::thread> th;
    for (uint32_t t = 0; t < std::min(threads, n); t++)
        th.emplace_back([&] {
            for (uint32_t i; (i = next.fetch_add(1)) < n;) fn(i);
        });
    for (auto& t : th) t.join();
}

}  // namespace

// ---------------------------------------------------------------------------
TerrainField::TerrainField(const TerrainParams& p) : p_(p), L_(1u << p.depth) {
    band_ = p.variant != 0 ? 16.0f : 0.0f;
    heights_.resize(size_t(L_) * L_);
    const uint32_t sh = seed32(p.seed, 0x4845u);
    for (uint32_t z = 0; z < L_; z++)
        for (uint32_t x = 0; x < L_; x++)
            heights_[size_t(z) * L_ + x] =
                float(64.0 + 32.0 * fbm2((x + 0.5) / 32.0, (z + 0.5) / 32.0, 4, sh));
    if (p.variant == 2 && L_ > 1024u) {  // island: columns outside the central 1024 x 1024 hold nothing
        const uint32_t lo = (L_ - 1024u) / 2u;
        for (uint32_t z = 0; z < L_; z++)
            for (uint32_t x = 0; x < L_; x++)
                if (x < lo || z < lo || x >= lo + 1024u || z >= lo + 1024u) heights_[size_t(z) * L_ + x] = -1.0e6f;
    }
}

bool TerrainField::solid(uint32_t x, uint32_t y, uint32_t z) const {
    const double yc = double(y) + 0.5;
    const double h = double(height(x, z));
    if (p_.variant == 0) return yc < h;
    const double A = band_;
    if (yc < h - A) return true;
    if (yc >= h + A) return false;
    const double f = fbm3((x + 0.5) / 24.0, yc / 24.0, (z + 0.5) / 24.0, 3, seed32(p_.seed, 0x4f56u));
    return yc < h + A * f;
}

uint32_t TerrainField::material(uint32_t x, uint32_t y, uint32_t z) const {
    const uint32_t s = seed32(p_.seed, 0x4d41u);
    return 1u + mix32(x * 0x9E3779B1u ^ mix32(y * 0x85EBCA77u ^ mix32(z * 0xC2B2AE3Du ^ s))) % 8u;
}

std::vector<uint32_t> terrain_voxels(const TerrainParams& p) {
    TerrainField f(p);
    const uint32_t L = f.length();
    // no voxel is solid at or above the highest column top plus the band
    double top = 0.0;
    for (uint32_t z = 0; z < L; z++)
        for (uint32_t x = 0; x < L; x++) top = std::max(top, double(f.height(x, z)));
    const uint32_t ymax = uint32_t(std::min<double>(L, std::max(0.0, std::ceil(top + f.band())) + 1.0));
    std::vector<uint32_t> out;
    for (uint32_t x = 0; x < L; x++)
        for (uint32_t y = 0; y < ymax; y++)
            for (uint32_t z = 0; z < L; z++)
                if (f.solid(x, y, z)) {
                    out.push_back(x);
                    out.push_back(y);
                    out.push_back(z);
                    out.push_back(f.material(x, y, z));
                }
    return out;
}

// ---------------------------------------------------------------------------
namespace {

struct Pyramid {
    uint32_t D;
    uint32_t nb;                          // bricks per axis (2^(D-3))
    std::vector<uint64_t> bits;           // 8 words per brick: bit (lx<<6)|(ly<<3)|lz
    std::vector<uint64_t> m2;             // occupied 2^3 sub-cubes: bit (sx<<4)|(sy<<2)|sz, s in [0,4)
    std::vector<uint8_t> m4;              // occupied 4^3 sub-cubes: bit (sx<<2)|(sy<<1)|sz
    std::vector<std::vector<uint8_t>> occ;  // levels 0..D-3: 1 byte per cell

    static size_t lin(uint32_t x, uint32_t y, uint32_t z, uint32_t n) { return (size_t(x) * n + y) * n + z; }

    bool occupied(uint32_t k, uint32_t x, uint32_t y, uint32_t z) const {
        if (k + 3 <= D) return occ[k][lin(x, y, z, 1u << k)] != 0;
        if (k + 2 == D) {
            const size_t b = lin(x >> 1, y >> 1, z >> 1, nb);
            return (m4[b] >> (((x & 1) << 2) | ((y & 1) << 1) | (z & 1))) & 1u;
        }
        if (k + 1 == D) {
            const size_t b = lin(x >> 2, y >> 2, z >> 2, nb);
            return (m2[b] >> (((x & 3) << 4) | ((y & 3) << 2) | (z & 3))) & 1u;
        }
        const size_t b = lin(x >> 3, y >> 3, z >> 3, nb);
        const uint32_t l = ((x & 7) << 6) | ((y & 7) << 3) | (z & 7);
        return (bits[b * 8 + (l >> 6)] >> (l & 63)) & 1u;
    }

    // internal nodes (occupied cells of size >= 2) in the subtree of an
    // occupied cell at level k, the cell included
    uint64_t count_internal(uint32_t k, uint32_t x, uint32_t y, uint32_t z) const {
        if (k >= D) return 0;
        if (k + 1 == D) return 1;
        if (k + 3 == D) {
            const size_t b = lin(x, y, z, nb);
            return 1u + uint64_t(__builtin_popcount(m4[b])) + uint64_t(__builtin_popcountll(m2[b]));
        }
        if (k + 2 == D) {
            const size_t b = lin(x >> 1, y >> 1, z >> 1, nb);
            const uint32_t sx = (x & 1) * 2, sy = (y & 1) * 2, sz = (z & 1) * 2;
            uint64_t c = 1;
            for (uint32_t i = 0; i < 8; i++) {
                const uint32_t a = sx + ((i >> 2) & 1), bb = sy + ((i >> 1) & 1), cc = sz + (i & 1);
                c += (m2[b] >> ((a << 4) | (bb << 2) | cc)) & 1u;
            }
            return c;
        }
        uint64_t c = 1;
        for (uint32_t i = 0; i < 8; i++) {
            const uint32_t cx = 2 * x + ((i >> 2) & 1), cy = 2 * y + ((i >> 1) & 1), cz = 2 * z + (i & 1);
            if (occupied(k + 1, cx, cy, cz)) c += count_internal(k + 1, cx, cy, cz);
        }
        return c;
    }
};

struct Emitter {
    const Pyramid& P;
    const TerrainField& F;
    uint32_t* data;
    uint64_t nvox = 0;

    // DFS pre-order, children 7..0 (linearizeNode's LIFO order)
    void emit(uint32_t k, uint32_t x, uint32_t y, uint32_t z, uint32_t slot, uint32_t& cursor) {
        if (k == P.D) {
            data[slot] = make_leaf_word(F.material(x, y, z));
            nvox++;
            return;
        }
        const uint32_t block = cursor;
        cursor += 8;
        uint32_t count = 0;
        for (uint32_t i = 0; i < 8; i++)
            count += P.occupied(k + 1, 2 * x + ((i >> 2) & 1), 2 * y + ((i >> 1) & 1), 2 * z + (i & 1));
        data[slot] = make_internal_word(count, block);
        for (int i = 7; i >= 0; i--) {
            const uint32_t cx = 2 * x + ((i >> 2) & 1), cy = 2 * y + ((i >> 1) & 1), cz = 2 * z + (i & 1);
            if (P.occupied(k + 1, cx, cy, cz)) emit(k + 1, cx, cy, cz, block + uint32_t(i), cursor);
        }
    }
};

}  // namespace

std::vector<uint32_t> build_terrain_words(const TerrainParams& p, uint32_t threads, uint64_t* n_voxels) {
    if (threads == 0) threads = std::max(1u, std::thread::hardware_concurrency());
    TerrainField F(p);
    const uint32_t D = p.depth;
    if (D < 4) {  // tiny scenes: the pointer tree path
        OctreeCPU cpu{uint8_t(D)};
        std::vector<uint32_t> v = terrain_voxels(p);
        for (size_t i = 0; i < v.size(); i += 4) cpu.insert(v[i], v[i + 1], v[i + 2], v[i + 3]);
        Octree o{uint8_t(D)};
        o.set(&cpu);
        if (n_voxels) *n_voxels = o.numVoxels;
        return std::vector<uint32_t>(o.data.begin(), o.data.begin() + (cpu.root ? o.size : 9));
    }
    Pyramid P;
    P.D = D;
    P.nb = 1u << (D - 3);
    const uint32_t nb = P.nb;
    const size_t nbricks = size_t(nb) * nb * nb;
    P.bits.assign(nbricks * 8, 0ull);
    P.m2.assign(nbricks, 0ull);
    P.m4.assign(nbricks, 0u);
    P.occ.resize(D - 2);
    P.occ[D - 3].assign(nbricks, 0u);
    const double A = F.band();
    // 1. bricks
    parallel_for(nb, threads, [&](uint32_t bx) {
        for (uint32_t bz = 0; bz < nb; bz++) {
            double hmin = 1e30, hmax = -1e30;
            for (uint32_t lx = 0; lx < 8; lx++)
                for (uint32_t lz = 0; lz < 8; lz++) {
                    const double h = F.height(bx * 8 + lx, bz * 8 + lz);
                    hmin = std::min(hmin, h);
                    hmax = std::max(hmax, h);
                }
            for (uint32_t by = 0; by < nb; by++) {
                const size_t b = Pyramid::lin(bx, by, bz, nb);
                uint64_t* w = &P.bits[b * 8];
                const double y0 = by * 8.0 + 0.5, y1 = by * 8.0 + 7.5;
                if (y0 >= hmax + A) continue;  // every voxel above the band: empty
                if (y1 < hmin - A) {           // every voxel below the band: solid
                    for (int i = 0; i < 8; i++) w[i] = ~0ull;
                } else {
                    for (uint32_t lx = 0; lx < 8; lx++)
                        for (uint32_t ly = 0; ly < 8; ly++)
                            for (uint32_t lz = 0; lz < 8; lz++)
                                if (F.solid(bx * 8 + lx, by * 8 + ly, bz * 8 + lz)) {
                                    const uint32_t l = (lx << 6) | (ly << 3) | lz;
                                    w[l >> 6] |= 1ull << (l & 63);
                                }
                }
                uint64_t m2 = 0;
                for (uint32_t v = 0; v < 512; v++) {
                    if (!((w[v >> 6] >> (v & 63)) & 1u)) continue;
                    const uint32_t lx = v >> 6, ly = (v >> 3) & 7, lz = v & 7;
                    m2 |= 1ull << (((lx >> 1) << 4) | ((ly >> 1) << 2) | (lz >> 1));
                }
                uint8_t m4 = 0;
                for (uint32_t s = 0; s < 64; s++) {
                    if (!((m2 >> s) & 1u)) continue;
                    const uint32_t sx = s >> 4, sy = (s >> 2) & 3, sz = s & 3;
                    m4 |= uint8_t(1u << (((sx >> 1) << 2) | ((sy >> 1) << 1) | (sz >> 1)));
                }
                P.m2[b] = m2;
                P.m4[b] = m4;
                P.occ[D - 3][b] = m4 != 0;
            }
        }
    });
    // 2. pyramid above bricks
    for (int k = int(D) - 4; k >= 0; k--) {
        const uint32_t n = 1u << k;
        P.occ[k].assign(size_t(n) * n * n, 0u);
        for (uint32_t x = 0; x < n; x++)
            for (uint32_t y = 0; y < n; y++)
                for (uint32_t z = 0; z < n; z++) {
                    uint8_t o = 0;
                    for (uint32_t i = 0; i < 8; i++)
                        o |= P.occ[k + 1][Pyramid::lin(2 * x + ((i >> 2) & 1), 2 * y + ((i >> 1) & 1),
                                                       2 * z + (i & 1), n * 2)];
                    P.occ[k][Pyramid::lin(x, y, z, n)] = o;
                }
    }
    if (!P.occ[0][0]) {
        if (n_voxels) *n_voxels = 0;
        return std::vector<uint32_t>(9, 0u);
    }
    // 3. block bases: root children in order 0..7, each followed by its
    //    children's subtrees in order 7..0
    uint32_t rootCount = 0;
    for (uint32_t c = 0; c < 8; c++) rootCount += P.occupied(1, (c >> 2) & 1, (c >> 1) & 1, c & 1);
    struct Task {
        uint32_t x, y, z, slot, base;
    };
    std::vector<Task> tasks;
    uint64_t cursor = 9;
    uint32_t rootBlock[8];
    for (uint32_t c = 0; c < 8; c++) {
        const uint32_t x1 = (c >> 2) & 1, y1 = (c >> 1) & 1, z1 = c & 1;
        if (!P.occupied(1, x1, y1, z1)) continue;
        rootBlock[c] = uint32_t(cursor);
        cursor += 8;
        for (int j = 7; j >= 0; j--) {
            const uint32_t x2 = 2 * x1 + ((j >> 2) & 1), y2 = 2 * y1 + ((j >> 1) & 1), z2 = 2 * z1 + (j & 1);
            if (!P.occupied(2, x2, y2, z2)) continue;
            tasks.push_back({x2, y2, z2, rootBlock[c] + uint32_t(j), uint32_t(cursor)});
            cursor += 8ull * P.count_internal(2, x2, y2, z2);
        }
    }
    if (cursor > (1ull << 28)) {
        if (n_voxels) *n_voxels = 0;
        return {};  // does not fit the 28-bit `next` field
    }
    std::vector<uint32_t> data(cursor, 0u);
    data[0] = make_internal_word(rootCount, 1);
    for (uint32_t c = 0; c < 8; c++) {
        const uint32_t x1 = (c >> 2) & 1, y1 = (c >> 1) & 1, z1 = c & 1;
        if (!P.occupied(1, x1, y1, z1)) continue;
        uint32_t cnt = 0;
        for (uint32_t i = 0; i < 8; i++)
            cnt += P.occupied(2, 2 * x1 + ((i >> 2) & 1), 2 * y1 + ((i >> 1) & 1), 2 * z1 + (i & 1));
        data[1 + c] = make_internal_word(cnt, rootBlock[c]);
    }
    std::vector<uint64_t> nv(tasks.size(), 0);
    parallel_for(uint32_t(tasks.size()), threads, [&](uint32_t t) {
        Emitter e{P, F, data.data()};
        uint32_t cur = tasks[t].base;
        e.emit(2, tasks[t].x, tasks[t].y, tasks[t].z, tasks[t].slot, cur);
        nv[t] = e.nvox;
    });
    uint64_t total = 0;
    for (uint64_t v : nv) total += v;
    if (n_voxels) *n_voxels = total;
    return data;
}

// ---------------------------------------------------------------------------
void camera_ubo(const float pos[3], const float dir[3], float fov_deg, float aspect, float ubo[16]) {
    // glm semantics: normalize(v) = v * inversesqrt(dot(v, v)),
    // radians(x) = x * 0.01745329251994329576923690768489
    auto norm = [](const float v[3], float o[3]) {
        const float is = 1.0f / std::sqrt((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]);
        o[0] = v[0] * is; o[1] = v[1] * is; o[2] = v[2] * is;
    };
    auto cross = [](const float a[3], const float b[3], float o[3]) {
        o[0] = a[1] * b[2] - b[1] * a[2];
        o[1] = a[2] * b[0] - b[2] * a[0];
        o[2] = a[0] * b[1] - b[0] * a[1];
    };
    const float tn = std::tan((fov_deg / 2.0f) * 0.01745329251994329576923690768489f);
    const float Y[3] = {0.0f, 1.0f, 0.0f};
    float c[3], r[3], u[3], n[3];
    cross(Y, dir, c);
    norm(c, n);
    for (int i = 0; i < 3; i++) r[i] = n[i] * tn * aspect;
    cross(r, dir, c);
    norm(c, n);
    for (int i = 0; i < 3; i++) u[i] = n[i] * tn;
    const float v[16] = {pos[0], pos[1], pos[2], 0.0f, dir[0], dir[1], dir[2], 0.0f,
                         r[0],   r[1],   r[2],   0.0f, u[0],   u[1],   u[2],   0.0f};
    std::memcpy(ubo, v, sizeof(v));
}

void terrain_materials(uint64_t seed, MaterialStd140 out[128]) {
    std::memset(out, 0, sizeof(MaterialStd140) * 128);
    uint64_t s = seed ^ 0x6d6174657269616cull;
    for (int i = 1; i <= 8; i++) {
        for (int c = 0; c < 3; c++) {
            const double u = double(splitmix64(s) >> 11) * (1.0 / 9007199254740992.0);
            out[i].color[c] = float(0.2 + 0.7 * u);
            out[i].specularColor[c] = out[i].color[c];
        }
        out[i].color[3] = 0.0f;
        out[i].specularColor[3] = 1.0f;
        out[i].roughness = 1.0f;
        out[i].specular = 0.0f;
        out[i].metallic = 0.0f;
        out[i].emissive = 0;
        out[i].emissiveIntensity = 0.0f;
    }
}

}  // namespace ve
