// host_api.cpp — C ABI over the host scene layer (include/ve.h, "Host scene
// layer" section): OctreeCPU, Octree, terrain scenes, camera basis.
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../../include/ve.h"
#include "scene_host.h"

struct ve_octree_cpu {
    ve::OctreeCPU t;
    explicit ve_octree_cpu(uint8_t d) : t(d) {}
};
struct ve_octree {
    ve::Octree o;
    std::vector<uint32_t> changed;
    explicit ve_octree(uint8_t d) : o(d) {}
};
struct ve_words {
    std::vector<uint32_t> w;
};

namespace ve {
void set_last_error(const char* msg);  // render.cu: one per-thread message for the whole ABI
}
namespace {
int hfail(int code, const char* msg) {
    ve::set_last_error(msg);
    return code;
}
}  // namespace

extern "C" {

const char* ve_version(void) { return "voxelengine3.0-b200 1.0 (sm_100a)"; }

int ve_octree_cpu_create(uint32_t depth, ve_octree_cpu** out) {
    if (!out) return hfail(VE_ERR_INVALID, "octree_cpu_create: null output");
    if (depth < 1 || depth > 16) return hfail(VE_ERR_INVALID, "octree_cpu_create: depth must be in [1, 16]");
    *out = new ve_octree_cpu(uint8_t(depth));
    return VE_OK;
}
int ve_octree_cpu_destroy(ve_octree_cpu* t) {
    delete t;
    return VE_OK;
}
int ve_octree_cpu_insert(ve_octree_cpu* t, uint32_t x, uint32_t y, uint32_t z, uint32_t m) {
    if (!t) return hfail(VE_ERR_INVALID, "insert: null tree");
    t->t.insert(x, y, z, m);
    return VE_OK;
}
int ve_octree_cpu_insert_many(ve_octree_cpu* t, const uint32_t* v, uint64_t n) {
    if (!t || (!v && n)) return hfail(VE_ERR_INVALID, "insert_many: null argument");
    for (uint64_t i = 0; i < n; i++) t->t.insert(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
    return VE_OK;
}
int ve_octree_cpu_remove(ve_octree_cpu* t, uint32_t x, uint32_t y, uint32_t z) {
    if (!t) return hfail(VE_ERR_INVALID, "remove: null tree");
    t->t.remove(x, y, z);
    return VE_OK;
}
int ve_octree_cpu_lookup(const ve_octree_cpu* t, uint32_t x, uint32_t y, uint32_t z, int64_t* m) {
    if (!t || !m) return hfail(VE_ERR_INVALID, "lookup: null argument");
    ve::OctreeCPU::Node* n = t->t.lookup(x, y, z);
    *m = n ? int64_t(n->material) : -1;
    return VE_OK;
}
int ve_octree_cpu_insert_box(ve_octree_cpu* t, const uint32_t mn[3], const uint32_t mx[3], uint32_t m) {
    if (!t || !mn || !mx) return hfail(VE_ERR_INVALID, "insert_box: null argument");
    t->t.insertBox(mn, mx, m);
    return VE_OK;
}
int ve_octree_cpu_insert_sphere(ve_octree_cpu* t, const float c[3], float r, uint32_t m) {
    if (!t || !c) return hfail(VE_ERR_INVALID, "insert_sphere: null argument");
    t->t.insertSphere(c, r, m);
    return VE_OK;
}
int ve_octree_cpu_raycast(const ve_octree_cpu* t, const float o[3], const float d[3], uint32_t max_steps, int* hit,
                          uint32_t pos[3]) {
    if (!t || !o || !d || !hit) return hfail(VE_ERR_INVALID, "raycast: null argument");
    ve::OctreeCPU::RayHit h = t->t.raycast(o, d, max_steps);
    *hit = h.hit ? 1 : 0;
    if (pos) std::memcpy(pos, h.position, sizeof(h.position));
    return VE_OK;
}

int ve_octree_create(uint32_t depth, ve_octree** out) {
    if (!out) return hfail(VE_ERR_INVALID, "octree_create: null output");
    if (depth < 1 || depth > 16) return hfail(VE_ERR_INVALID, "octree_create: depth must be in [1, 16]");
    *out = new ve_octree(uint8_t(depth));
    return VE_OK;
}
int ve_octree_destroy(ve_octree* o) {
    delete o;
    return VE_OK;
}
int ve_octree_set(ve_octree* o, ve_octree_cpu* c) {
    if (!o || !c) return hfail(VE_ERR_INVALID, "octree_set: null argument");
    o->o.set(&c->t);
    return VE_OK;
}
int ve_octree_apply_edits(ve_octree* o, ve_octree_cpu* c, uint32_t* changed, uint64_t cap, uint64_t* n) {
    if (!o || !c) return hfail(VE_ERR_INVALID, "apply_edits: null argument");
    o->changed.clear();
    o->o.applyEdits(&c->t, &o->changed);
    if (n) *n = o->changed.size();
    if (changed)
        for (uint64_t i = 0; i < o->changed.size() && i < cap; i++) changed[i] = o->changed[i];
    return VE_OK;
}
int ve_octree_last_changed(const ve_octree* o, const uint32_t** slots, uint64_t* n) {
    if (!o || !slots || !n) return hfail(VE_ERR_INVALID, "last_changed: null argument");
    *slots = o->changed.data();
    *n = o->changed.size();
    return VE_OK;
}
int ve_octree_find_gpu_slot(const ve_octree* o, ve_octree_cpu* c, uint32_t x, uint32_t y, uint32_t z,
                            uint32_t* slot) {
    if (!o || !c || !slot) return hfail(VE_ERR_INVALID, "find_gpu_slot: null argument");
    const uint32_t p[3] = {x, y, z};
    *slot = o->o.findGpuSlot(&c->t, p);
    return VE_OK;
}
int ve_octree_info(const ve_octree* o, uint32_t* size, uint32_t* capacity, uint32_t* nv) {
    if (!o) return hfail(VE_ERR_INVALID, "octree_info: null octree");
    if (size) *size = o->o.size;
    if (capacity) *capacity = o->o.capacity;
    if (nv) *nv = o->o.numVoxels;
    return VE_OK;
}
int ve_octree_words(const ve_octree* o, const uint32_t** w, uint64_t* n) {
    if (!o || !w || !n) return hfail(VE_ERR_INVALID, "octree_words: null argument");
    *w = o->o.data.data();
    *n = o->o.data.size();
    return VE_OK;
}

int ve_terrain_build(uint32_t depth, uint32_t variant, uint64_t seed, uint32_t threads, ve_words** out,
                     uint64_t* n_voxels) {
    if (!out) return hfail(VE_ERR_INVALID, "terrain_build: null output");
    if (depth < 1 || depth > 11) return hfail(VE_ERR_INVALID, "terrain_build: depth must be in [1, 11]");
    if (variant > 2) return hfail(VE_ERR_INVALID, "terrain_build: variant must be 0, 1 or 2");
    ve_words* w = new ve_words();
    w->w = ve::build_terrain_words(ve::TerrainParams{depth, variant, seed}, threads, n_voxels);
    if (w->w.empty()) {
        delete w;
        return hfail(VE_ERR_CAPACITY, "terrain_build: node array exceeds 2^28 words");
    }
    *out = w;
    return VE_OK;
}
int ve_words_data(const ve_words* w, const uint32_t** d, uint64_t* n) {
    if (!w || !d || !n) return hfail(VE_ERR_INVALID, "words_data: null argument");
    *d = w->w.data();
    *n = w->w.size();
    return VE_OK;
}
int ve_words_free(ve_words* w) {
    delete w;
    return VE_OK;
}
int ve_terrain_voxels(uint32_t depth, uint32_t variant, uint64_t seed, uint32_t* xyzm, uint64_t cap, uint64_t* n) {
    if (depth < 1 || depth > 10) return hfail(VE_ERR_INVALID, "terrain_voxels: depth must be in [1, 10]");
    std::vector<uint32_t> v = ve::terrain_voxels(ve::TerrainParams{depth, variant, seed});
    if (n) *n = v.size() / 4;
    if (xyzm) std::memcpy(xyzm, v.data(), std::min<uint64_t>(cap, v.size() / 4) * 16);
    return VE_OK;
}
int ve_terrain_materials(uint64_t seed, void* out) {
    if (!out) return hfail(VE_ERR_INVALID, "terrain_materials: null output");
    ve::terrain_materials(seed, static_cast<ve::MaterialStd140*>(out));
    return VE_OK;
}
int ve_camera_ubo(const float pos[3], const float dir[3], float fov, float aspect, float ubo[16]) {
    if (!pos || !dir || !ubo) return hfail(VE_ERR_INVALID, "camera_ubo: null argument");
    ve::camera_ubo(pos, dir, fov, aspect, ubo);
    return VE_OK;
}

}  // extern "C"
