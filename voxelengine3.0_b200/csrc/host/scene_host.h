// scene_host.h — host-side scene layer of the B200 voxel ray pipeline.
//
// Keeps the reference's scene API and GPU node layout:
//   * OctreeCPU: pointer sparse voxel octree with the reference's build/insert
//     API (src/octree_cpu.hpp:9-57).
//   * Octree: the 32-bit node array in the reference's linearisation order
//     (src/renderer/octree.hpp:14-98, octree.cpp:127-341), the exact words
//     the device traversal reads.
//   * TerrainBuilder: a parallel bulk builder that emits the same words as
//     OctreeCPU::insert + Octree::set for the seeded value-noise terrain
//     scenes, without building pointer nodes.
//   * camera basis (src/renderer/camera.cpp:39-50) and material table
//     (src/renderer/material.hpp:17-25).
#pragma once
#include <cstdint>
#include <functional>
#include <stack>
#include <vector>

namespace ve {

// Node word fields (src/renderer/octree.hpp:16-37):
//   internal: bit0 = 1, bits1-3 childrenCount (mod 8), bits4-31 next block
//   leaf:     bit0 = 0, bits1-7 material, bits8-31 normal field
inline uint32_t make_internal_word(uint32_t count, uint32_t next) {
    return 1u | ((count & 7u) << 1) | (next << 4);
}
inline uint32_t make_leaf_word(uint32_t material) { return (material & 0x7Fu) << 1; }

class OctreeCPU {
public:
    struct Node {
        Node* children[8] = {};
        uint8_t childrenCount = 0;
        uint32_t material = 0;
        uint32_t gpuBlock = UINT32_MAX;  // start of this node's 8-child block in Octree::data
        bool dirty = false;              // cleared by Octree::set / applyEdits
    };
    struct RayHit {
        bool hit = false;
        Node* node = nullptr;
        uint32_t position[3] = {0, 0, 0};
    };

    explicit OctreeCPU(uint8_t depth);
    ~OctreeCPU();
    OctreeCPU(const OctreeCPU&) = delete;
    OctreeCPU& operator=(const OctreeCPU&) = delete;

    RayHit raycast(const float origin[3], const float direction[3], uint32_t maxSteps = 300) const;
    void insert(uint32_t x, uint32_t y, uint32_t z, uint32_t material);
    void remove(uint32_t x, uint32_t y, uint32_t z);
    Node* lookup(uint32_t x, uint32_t y, uint32_t z) const;
    void insertBox(const uint32_t mn[3], const uint32_t mx[3], uint32_t material);
    void insertSphere(const float centre[3], float radius, uint32_t material);
    void insertFunction(const std::function<bool(float, float, float)>& fn, const uint32_t mn[3],
                        const uint32_t mx[3], uint32_t material);

    Node* root = nullptr;
    uint8_t depth = 0;
    std::vector<uint32_t> freedGpuBlocks;  // blocks released by remove() since the last applyEdits

private:
    uint32_t p2r_[18] = {};
    uint32_t locate(uint32_t x, uint32_t y, uint32_t z, uint32_t level) const;
    Node* alloc();
    void release(Node* n);
    void removeR(uint32_t x, uint32_t y, uint32_t z, Node*& node, uint32_t level);
    std::vector<Node*> chunks_;
    std::vector<Node*> free_;
};

class Octree {
public:
    explicit Octree(uint8_t depth);

    // Full linearisation (Octree::set, src/renderer/octree.cpp:127-217).
    void set(OctreeCPU* cpu);
    // Incremental resync of dirty nodes (octree.cpp:228-314); the slots whose
    // words changed are appended to `changed` (duplicates possible).
    void applyEdits(OctreeCPU* cpu, std::vector<uint32_t>* changed = nullptr);
    // GPU slot of the leaf at pos or UINT32_MAX (octree.cpp:322-341).
    uint32_t findGpuSlot(OctreeCPU* cpu, const uint32_t pos[3]) const;

    std::vector<uint32_t> data;  // `capacity` words; [size, capacity) are zero
    uint8_t depth;
    uint32_t capacity = 8;
    uint32_t size = 8;
    uint32_t numVoxels = 0;
    uint32_t maxWords = 1u << 28;  // `next` has 28 bits (octree.hpp:23)

private:
    std::stack<uint32_t> freeBlocks_;
    void resizeIfNeeded(uint32_t required);
    void applyEditsNode(OctreeCPU* cpu, OctreeCPU::Node* node, uint32_t slot, uint32_t level,
                        std::vector<uint32_t>* changed);
};

// Seeded value-noise terrain used by the benchmark scenes.
//   variant 0 ("small"): solid iff y+0.5 < 64 + 32*fBm2((x+0.5)/32, (z+0.5)/32)
//       with 4 octaves, gain 0.5, lacunarity 2 (fBm normalised to [-1, 1]).
//   variant 1 ("overhang"): the same heightfield plus 3 octaves of 3D value
//       noise: solid iff y+0.5 < h(x,z) + 16*fBm3((x,y,z)+0.5)/24) — carves
//       overhangs and caves within +-16 voxels of the surface.
//   variant 2 ("island"): variant 1 restricted to the central 1024 x 1024
//       columns (the whole scene up to depth 10).  A depth-11 scene of this
//       family: the full-extent terrain at depth 11 holds ~270M solid voxels,
//       more leaf slots than the layout's 28-bit `next` field addresses.
// material = 1 + (hash(x, y, z, seed) mod 8).
struct TerrainParams {
    uint32_t depth;
    uint32_t variant;
    uint64_t seed;
};

class TerrainField {
public:
    explicit TerrainField(const TerrainParams& p);
    bool solid(uint32_t x, uint32_t y, uint32_t z) const;
    uint32_t material(uint32_t x, uint32_t y, uint32_t z) const;
    float height(uint32_t x, uint32_t z) const { return heights_[size_t(z) * L_ + x]; }
    float band() const { return band_; }
    uint32_t length() const { return L_; }

private:
    TerrainParams p_;
    uint32_t L_;
    float band_;
    std::vector<float> heights_;
};

// Parallel bulk build of the terrain's node words in the exact order of
// OctreeCPU::insert + Octree::set.  Returns `size` words (no capacity
// padding); reports the voxel count.
std::vector<uint32_t> build_terrain_words(const TerrainParams& p, uint32_t threads, uint64_t* n_voxels);

// Every solid voxel of the terrain as (x, y, z, material), x-major order.
std::vector<uint32_t> terrain_voxels(const TerrainParams& p);

// Camera::UpdateUBO (src/renderer/camera.cpp:39-50).
void camera_ubo(const float pos[3], const float dir[3], float fov_deg, float aspect, float ubo[16]);

// Material table entry (std140, 64 B; src/renderer/material.hpp:17-25).
struct MaterialStd140 {
    float color[4];
    float specularColor[4];
    float roughness, specular, metallic;
    int32_t emissive;
    float emissiveIntensity;
    float pad[3];
};
static_assert(sizeof(MaterialStd140) == 64, "std140 material stride");

// 128-entry table: slot 0 reserved; slots 1..8 Lambertian with albedo
// U[0.2, 0.9]^3 from `seed`, roughness 1, metallic 0, specular 0.
void terrain_materials(uint64_t seed, MaterialStd140 out[128]);

}  // namespace ve
