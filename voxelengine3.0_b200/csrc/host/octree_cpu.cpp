// octree_cpu.cpp — OctreeCPU (pointer SVO) and Octree (reference node layout).
//
// API and semantics follow the reference: src/octree_cpu.cpp (insert :40-64,
// remove :66-98, lookup :100-112, raycast :128-215, insertBox/Sphere/Function
// :221-262) and src/renderer/octree.cpp (set :127-166, linearizeNode :170-217,
// applyEdits :228-314, findGpuSlot :322-341).  The node word layout and the
// slot order are kept bit-for-bit; nodes come from a chunked free-list pool
// instead of one heap allocation each.
#include <cmath>
#include <tuple>

#include "scene_host.h"

namespace ve {

namespace {
constexpr size_t kChunk = 4096;
inline float fmin_g(float a, float b) { return (b < a) ? b : a; }
inline float fmax_g(float a, float b) { return (a < b) ? b : a; }
}  // namespace

OctreeCPU::OctreeCPU(uint8_t d) : depth(d) {
    uint32_t p = 1;
    for (int i = int(d); i >= 1; i--) {
        p2r_[i] = p;
        p <<= 1;
    }
    p2r_[0] = p;
}

OctreeCPU::~OctreeCPU() {
    for (Node* c : chunks_) delete[] c;
}

OctreeCPU::Node* OctreeCPU::alloc() {
    if (free_.empty()) {
        Node* c = new Node[kChunk];
        chunks_.push_back(c);
        for (size_t i = kChunk; i-- > 0;) free_.push_back(&c[i]);
    }
    Node* n = free_.back();
    free_.pop_back();
    *n = Node();
    return n;
}

void OctreeCPU::release(Node* n) { free_.push_back(n); }

uint32_t OctreeCPU::locate(uint32_t x, uint32_t y, uint32_t z, uint32_t level) const {
    const uint32_t p2 = p2r_[level];
    return (uint32_t(bool(x & p2)) << 2) | (uint32_t(bool(y & p2)) << 1) | uint32_t(bool(z & p2));
}

void OctreeCPU::insert(uint32_t x, uint32_t y, uint32_t z, uint32_t material) {
    const uint32_t bound = 1u << depth;
    if (x >= bound || y >= bound || z >= bound) return;
    if (!root) root = alloc();
    Node* n = root;
    for (uint32_t level = 1; level <= depth; level++) {
        n->dirty = true;
        const uint32_t idx = locate(x, y, z, level);
        if (!n->children[idx]) {
            n->children[idx] = alloc();
            n->childrenCount++;
        }
        n = n->children[idx];
    }
    n->dirty = true;
    n->material = material;
    n->childrenCount = 0;
}

void OctreeCPU::remove(uint32_t x, uint32_t y, uint32_t z) {
    const uint32_t bound = 1u << depth;
    if (x >= bound || y >= bound || z >= bound) return;
    if (!root) return;
    removeR(x, y, z, root, 1);
}

// removeR (src/octree_cpu.cpp:74-98): a parent whose last child vanished is
// released too, and its GPU block is queued for Octree::applyEdits.
void OctreeCPU::removeR(uint32_t x, uint32_t y, uint32_t z, Node*& node, uint32_t level) {
    if (!node) return;
    node->dirty = true;
    if (level > depth) {
        release(node);
        node = nullptr;
        return;
    }
    const uint32_t idx = locate(x, y, z, level);
    const bool had = node->children[idx] != nullptr;
    removeR(x, y, z, node->children[idx], level + 1);
    if (had && node->children[idx] == nullptr) {
        node->childrenCount--;
        if (node->childrenCount == 0) {
            if (node->gpuBlock != UINT32_MAX) freedGpuBlocks.push_back(node->gpuBlock);
            release(node);
            node = nullptr;
        }
    }
}

OctreeCPU::Node* OctreeCPU::lookup(uint32_t x, uint32_t y, uint32_t z) const {
    const uint32_t bound = 1u << depth;
    if (x >= bound || y >= bound || z >= bound) return nullptr;
    Node* node = root;
    for (uint32_t level = 1; level <= uint32_t(depth) + 1; level++) {
        if (node == nullptr) return nullptr;
        if (level > depth) return node;
        node = node->children[locate(x, y, z, level)];
    }
    return nullptr;
}

// Same DDA as the device traversal but over pointers, with the reference's
// CPU step counting (no entry check, q <= maxSteps) and the FIXED advanced
// origin for every slab computation.
OctreeCPU::RayHit OctreeCPU::raycast(const float origin_in[3], const float dir[3], uint32_t maxSteps) const {
    RayHit none;
    if (!root) return none;
    const uint32_t L = 1u << depth;
    const float bF = float(L);
    const float inv[3] = {1.0f / dir[0], 1.0f / dir[1], 1.0f / dir[2]};
    float o[3];
    for (int c = 0; c < 3; c++) o[c] = origin_in[c] + dir[c] * 4.0f;
    auto inb = [&](const float p[3]) {
        return p[0] >= 0.0f && p[0] <= bF && p[1] >= 0.0f && p[1] <= bF && p[2] >= 0.0f && p[2] <= bF;
    };
    float r[3];
    if (inb(o)) {
        for (int c = 0; c < 3; c++) r[c] = o[c];
    } else {
        float tmi[3], tmx[3];
        for (int c = 0; c < 3; c++) {
            const float t1 = ((0.0f - o[c]) + 0.001f) * inv[c];
            const float t2 = ((bF - o[c]) - 0.001f) * inv[c];
            tmi[c] = fmin_g(t1, t2);
            tmx[c] = fmax_g(t1, t2);
        }
        const float te = fmax_g(fmax_g(tmi[0], tmi[1]), tmi[2]);
        const float tx = fmin_g(fmin_g(tmx[0], tmx[1]), tmx[2]);
        if (tx < te || tx < 0.0f) return none;
        for (int c = 0; c < 3; c++) r[c] = dir[c] * te + o[c];
    }
    for (uint32_t q = 0; inb(r) && q <= maxSteps; ++q) {
        const uint32_t u[3] = {uint32_t(r[0]), uint32_t(r[1]), uint32_t(r[2])};
        Node* node = root;
        uint32_t sz = L;
        uint32_t org[3] = {0, 0, 0};
        for (uint32_t lev = 1; lev <= depth; ++lev) {
            const uint32_t csz = 1u << (depth - lev);
            Node* ch = node->children[locate(u[0], u[1], u[2], lev)];
            const uint32_t co[3] = {u[0] & ~(csz - 1u), u[1] & ~(csz - 1u), u[2] & ~(csz - 1u)};
            if (!ch) {
                sz = csz ? csz : 1u;
                org[0] = co[0]; org[1] = co[1]; org[2] = co[2];
                break;
            }
            if (lev == depth) {
                if (ch->material != 0) {
                    RayHit h;
                    h.hit = true;
                    h.node = ch;
                    h.position[0] = u[0]; h.position[1] = u[1]; h.position[2] = u[2];
                    return h;
                }
                sz = 1u;
                org[0] = u[0]; org[1] = u[1]; org[2] = u[2];
                break;
            }
            node = ch;
            sz = csz;
            org[0] = co[0]; org[1] = co[1]; org[2] = co[2];
        }
        float tx = 0;
        for (int c = 0; c < 3; c++) {
            const float bmin = float(org[c]);
            const float bmax = bmin + float(sz);
            const float t1 = ((bmin - o[c]) - 0.001f) * inv[c];
            const float t2 = ((bmax - o[c]) + 0.001f) * inv[c];
            const float m = fmax_g(t1, t2);
            tx = c == 0 ? m : fmin_g(tx, m);
        }
        for (int c = 0; c < 3; c++) r[c] = dir[c] * tx + o[c];
    }
    return none;
}

void OctreeCPU::insertBox(const uint32_t mn[3], const uint32_t mx_in[3], uint32_t material) {
    const uint32_t bound = 1u << depth;
    uint32_t mx[3];
    for (int c = 0; c < 3; c++) mx[c] = mx_in[c] < bound ? mx_in[c] : bound;
    for (uint32_t x = mn[0]; x < mx[0]; x++)
        for (uint32_t y = mn[1]; y < mx[1]; y++)
            for (uint32_t z = mn[2]; z < mx[2]; z++) insert(x, y, z, material);
}

void OctreeCPU::insertSphere(const float c[3], float radius, uint32_t material) {
    const int32_t bound = int32_t(1u << depth);
    int32_t lo[3], hi[3];
    for (int k = 0; k < 3; k++) {
        const int32_t a = int32_t(std::floor(c[k] - radius));
        const int32_t b = int32_t(std::ceil(c[k] + radius));
        lo[k] = a > 0 ? a : 0;
        hi[k] = b < bound - 1 ? b : bound - 1;
    }
    for (int32_t x = lo[0]; x <= hi[0]; x++)
        for (int32_t y = lo[1]; y <= hi[1]; y++)
            for (int32_t z = lo[2]; z <= hi[2]; z++) {
                const float d0 = (float(x) + 0.5f) - c[0];
                const float d1 = (float(y) + 0.5f) - c[1];
                const float d2 = (float(z) + 0.5f) - c[2];
                if (std::sqrt((d0 * d0 + d1 * d1) + d2 * d2) <= radius) insert(uint32_t(x), uint32_t(y), uint32_t(z), material);
            }
}

void OctreeCPU::insertFunction(const std::function<bool(float, float, float)>& fn, const uint32_t mn[3],
                               const uint32_t mx_in[3], uint32_t material) {
    const uint32_t bound = 1u << depth;
    uint32_t mx[3];
    for (int c = 0; c < 3; c++) mx[c] = mx_in[c] < bound ? mx_in[c] : bound;
    for (uint32_t x = mn[0]; x < mx[0]; x++)
        for (uint32_t y = mn[1]; y < mx[1]; y++)
            for (uint32_t z = mn[2]; z < mx[2]; z++)
                if (fn(float(x) + 0.5f, float(y) + 0.5f, float(z) + 0.5f)) insert(x, y, z, material);
}

// ---------------------------------------------------------------------------
// Octree: reference node array
// ---------------------------------------------------------------------------
Octree::Octree(uint8_t d) : depth(d > 16 ? 16 : d) { data.assign(capacity, 0u); }

void Octree::resizeIfNeeded(uint32_t required) {
    if (required > capacity) {
        while (capacity < required) capacity *= 2;
        if (capacity > maxWords) capacity = maxWords;
        data.resize(capacity, 0u);
    }
}

void Octree::set(OctreeCPU* cpu) {
    if (!cpu || !cpu->root) return;
    data.assign(capacity, 0u);
    size = 9;
    numVoxels = 0;
    while (!freeBlocks_.empty()) freeBlocks_.pop();
    cpu->freedGpuBlocks.clear();
    resizeIfNeeded(size);
    cpu->root->gpuBlock = 1;
    cpu->root->dirty = false;
    data[0] = make_internal_word(cpu->root->childrenCount, 1);
    using Entry = std::tuple<OctreeCPU::Node*, uint32_t, uint32_t>;
    std::vector<Entry> st;
    for (uint32_t i = 0; i < 8; i++) {
        st.clear();
        st.emplace_back(cpu->root->children[i], i + 1, 2u);
        while (!st.empty()) {
            auto [cn, off, lv] = st.back();
            st.pop_back();
            if (!cn) continue;
            cn->dirty = false;
            if (lv > cpu->depth || (cn->material != 0 && cn->childrenCount == 0)) {
                if (cn->material == 0) continue;
                resizeIfNeeded(off + 1);
                data[off] = make_leaf_word(cn->material);
                numVoxels++;
            } else {
                resizeIfNeeded(off + 1);
                const uint32_t block = size;
                size += 8;
                resizeIfNeeded(size);
                cn->gpuBlock = block;
                data[off] = make_internal_word(cn->childrenCount, block);
                for (uint32_t k = 0; k < 8; k++) st.emplace_back(cn->children[k], block + k, lv + 1);
            }
        }
    }
}

void Octree::applyEdits(OctreeCPU* cpu, std::vector<uint32_t>* changed) {
    if (!cpu || !cpu->root) return;
    for (uint32_t b : cpu->freedGpuBlocks) freeBlocks_.push(b);
    cpu->freedGpuBlocks.clear();
    if (!cpu->root->dirty) return;
    data[0] = make_internal_word(cpu->root->childrenCount, 1);
    if (changed) changed->push_back(0);
    cpu->root->dirty = false;
    for (uint32_t i = 0; i < 8; i++) applyEditsNode(cpu, cpu->root->children[i], i + 1, 2, changed);
}

void Octree::applyEditsNode(OctreeCPU* cpu, OctreeCPU::Node* node, uint32_t slot, uint32_t level,
                            std::vector<uint32_t>* changed) {
    if (!node) {
        if (data[slot] != 0u) {
            data[slot] = 0u;
            if (changed) changed->push_back(slot);
        }
        return;
    }
    if (!node->dirty) return;
    node->dirty = false;
    if (level > cpu->depth || (node->material != 0 && node->childrenCount == 0)) {
        data[slot] = make_leaf_word(node->material);
        if (changed) changed->push_back(slot);
        if (node->material != 0) numVoxels++;
        if (node->gpuBlock != UINT32_MAX) {
            freeBlocks_.push(node->gpuBlock);
            node->gpuBlock = UINT32_MAX;
        }
        return;
    }
    if (node->gpuBlock == UINT32_MAX) {
        uint32_t block;
        if (!freeBlocks_.empty()) {
            block = freeBlocks_.top();
            freeBlocks_.pop();
            for (uint32_t i = 0; i < 8; i++) {
                data[block + i] = 0u;
                if (changed) changed->push_back(block + i);
            }
        } else {
            if (size + 8 > maxWords) return;
            block = size;
            size += 8;
            resizeIfNeeded(size);
        }
        node->gpuBlock = block;
    }
    data[slot] = make_internal_word(node->childrenCount, node->gpuBlock);
    if (changed) changed->push_back(slot);
    for (uint32_t i = 0; i < 8; i++) applyEditsNode(cpu, node->children[i], node->gpuBlock + i, level + 1, changed);
}

uint32_t Octree::findGpuSlot(OctreeCPU* cpu, const uint32_t pos[3]) const {
    if (!cpu || !cpu->root) return UINT32_MAX;
    OctreeCPU::Node* node = cpu->root;
    uint32_t block = 1u;
    const uint32_t L = 1u << depth;
    for (uint32_t level = 1; level <= depth; level++) {
        const uint32_t p2 = L >> level;
        const uint32_t idx = (uint32_t(bool(pos[0] & p2)) << 2) | (uint32_t(bool(pos[1] & p2)) << 1) |
                             uint32_t(bool(pos[2] & p2));
        const uint32_t slot = block + idx;
        OctreeCPU::Node* child = node->children[idx];
        if (!child) return UINT32_MAX;
        if (level == depth) return slot;
        if (child->gpuBlock == UINT32_MAX) return UINT32_MAX;
        block = child->gpuBlock;
        node = child;
    }
    return UINT32_MAX;
}

}  // namespace ve
