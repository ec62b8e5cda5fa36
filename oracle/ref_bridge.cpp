// ref_bridge.cpp — test infrastructure.  A thin extern "C" bridge over the
// reference's OWN compiled octree code (src/octree_cpu.cpp and
// src/renderer/octree.cpp, compiled in place from the reference tree by
// oracle/build_ref.sh against the project-written shims in oracle/ref_shim/).
// Output goes only to oracle/_ref/.  Used by tests to pin the oracle's and the
// product's octree build / linearisation / raycast against the reference.
#include <cstring>
#include <vector>

#include "octree_cpu.hpp"
#include "renderer/octree.hpp"

namespace {
struct RefScene {
    OctreeCPU* cpu = nullptr;
    Octree* gpu = nullptr;
};
}  // namespace

extern "C" {

void* ref_scene_new(uint32_t depth) {
    RefScene* s = new RefScene();
    s->cpu = new OctreeCPU(uint8_t(depth));
    // Octree::Octree deletes its Config argument (src/renderer/octree.cpp:7).
    s->gpu = new Octree(new Octree::Config{uint8_t(depth)});
    return s;
}

void ref_scene_free(void* h) {
    RefScene* s = static_cast<RefScene*>(h);
    delete s->gpu;
    delete s->cpu;
    delete s;
}

void ref_insert(void* h, uint32_t x, uint32_t y, uint32_t z, uint32_t material) {
    static_cast<RefScene*>(h)->cpu->insert(glm::uvec3(x, y, z), material);
}

void ref_insert_many(void* h, const uint32_t* xyzm, uint64_t n) {
    OctreeCPU* c = static_cast<RefScene*>(h)->cpu;
    for (uint64_t i = 0; i < n; i++)
        c->insert(glm::uvec3(xyzm[4 * i], xyzm[4 * i + 1], xyzm[4 * i + 2]), xyzm[4 * i + 3]);
}

void ref_remove(void* h, uint32_t x, uint32_t y, uint32_t z) {
    static_cast<RefScene*>(h)->cpu->remove(glm::uvec3(x, y, z));
}

void ref_insert_box(void* h, const uint32_t mn[3], const uint32_t mx[3], uint32_t material) {
    static_cast<RefScene*>(h)->cpu->insertBox(glm::uvec3(mn[0], mn[1], mn[2]),
                                              glm::uvec3(mx[0], mx[1], mx[2]), material);
}

void ref_insert_sphere(void* h, float cx, float cy, float cz, float r, uint32_t material) {
    static_cast<RefScene*>(h)->cpu->insertSphere(glm::vec3(cx, cy, cz), r, material);
}

// Returns the material of the leaf at (x,y,z), or -1 when the lookup yields null.
int64_t ref_lookup(void* h, uint32_t x, uint32_t y, uint32_t z) {
    OctreeCPU::Node* n = static_cast<RefScene*>(h)->cpu->lookup(glm::uvec3(x, y, z));
    return n ? int64_t(n->material) : -1;
}

// Octree::set (src/renderer/octree.cpp:127-166); copies up to `cap` words of
// Octree::data.  Returns the number of words in data (capacity) and reports
// size / numVoxels.
uint64_t ref_set(void* h, uint32_t* out, uint64_t cap, uint32_t* size_out, uint32_t* nvox_out) {
    RefScene* s = static_cast<RefScene*>(h);
    s->gpu->set(s->cpu);
    uint64_t n = s->gpu->data.size();
    uint64_t m = n < cap ? n : cap;
    for (uint64_t i = 0; i < m; i++) out[i] = s->gpu->data[i].raw;
    if (size_out) *size_out = s->gpu->size;
    if (nvox_out) *nvox_out = s->gpu->numVoxels;
    return n;
}

// Octree::applyEdits (src/renderer/octree.cpp:228-249), same copy-out contract.
uint64_t ref_apply_edits(void* h, uint32_t* out, uint64_t cap, uint32_t* size_out) {
    RefScene* s = static_cast<RefScene*>(h);
    s->gpu->applyEdits(s->cpu);
    uint64_t n = s->gpu->data.size();
    uint64_t m = n < cap ? n : cap;
    for (uint64_t i = 0; i < m; i++) out[i] = s->gpu->data[i].raw;
    if (size_out) *size_out = s->gpu->size;
    return n;
}

uint32_t ref_find_gpu_slot(void* h, uint32_t x, uint32_t y, uint32_t z) {
    RefScene* s = static_cast<RefScene*>(h);
    return s->gpu->findGpuSlot(s->cpu, glm::uvec3(x, y, z));
}

// OctreeCPU::raycast (src/octree_cpu.cpp:128-215).  Returns 1 on hit and
// writes the voxel position.
int ref_raycast(void* h, const float o[3], const float d[3], uint32_t max_steps, uint32_t pos_out[3]) {
    OctreeCPU::RayHit r = static_cast<RefScene*>(h)->cpu->raycast(
        glm::vec3(o[0], o[1], o[2]), glm::vec3(d[0], d[1], d[2]), max_steps);
    if (!r.hit) return 0;
    pos_out[0] = r.position.x;
    pos_out[1] = r.position.y;
    pos_out[2] = r.position.z;
    return 1;
}

}  // extern "C"
