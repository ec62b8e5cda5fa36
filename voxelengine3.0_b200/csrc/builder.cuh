// builder.cuh — GPU bulk octree builder (part of the render.cu translation
// unit): from a voxel list to the node words that OctreeCPU::insert followed
// by Octree::set produce (octree_cpu.cpp:33-64, octree.cpp:127-217), bit for
// bit, without pointer nodes.
//
// 1. Morton keys: the child index at each level is (x bit << 2) | (y bit << 1)
//    | z bit (locate, internal.glsl:30), most significant level first, so a
//    stable key sort puts every subtree in one contiguous run with children
//    in index order.  Duplicate positions keep the last listed voxel, as
//    repeated inserts overwrite.
// 2. Levels bottom-up: the internal nodes of level l are the distinct key
//    prefixes of l-1 digits (root = level 1, voxels = level depth+1);
//    childrenCount = the number of distinct child prefixes under each.
// 3. Slots: Octree::set gives the root the block at slot 1 and then, per
//    root child in index order, walks a stack (children pushed 0..7, popped
//    7..0), allocating the next 8-slot block to every internal node it pops.
//    That is pre-order with the digits below the root child reversed; each
//    internal node's position in it is its rank under the 64-bit key
//    digit1+1, 8-digit2, 8-digit3, ... (4 bits each, zero padding sorts a
//    prefix before its extensions), and its block is 9 + 8 * rank.
// 4. Words: internal = 1 | (count & 7) << 1 | block << 4 at the slot
//    parent block + digit; leaves = (material & 0x7F) << 1.
#pragma once
#include <cub/cub.cuh>

namespace ve {
namespace build {

__device__ __forceinline__ uint64_t morton(uint32_t x, uint32_t y, uint32_t z, uint32_t D) {
    uint64_t k = 0;
    for (int b = int(D) - 1; b >= 0; b--)
        k = (k << 3) | (uint64_t((x >> b) & 1u) << 2) | (uint64_t((y >> b) & 1u) << 1) | uint64_t((z >> b) & 1u);
    return k;
}

__global__ void k_keys(const uint32_t* __restrict__ xyzm, uint64_t n, uint32_t D, uint64_t* __restrict__ keys,
                       uint32_t* __restrict__ idx) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        keys[i] = morton(xyzm[4 * i], xyzm[4 * i + 1], xyzm[4 * i + 2], D);
        idx[i] = uint32_t(i);
    }
}

// keep the last voxel of each run of equal keys
__global__ void k_last_of_run(const uint64_t* __restrict__ keys, uint64_t n, uint8_t* __restrict__ flag) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
        flag[i] = (i + 1 == n || keys[i] != keys[i + 1]) ? 1u : 0u;
}

// prefix of `shift` fewer bits; flag where it differs from the previous one
__global__ void k_prefix_heads(const uint64_t* __restrict__ in, uint64_t n, uint32_t shift, uint64_t* __restrict__ out,
                               uint32_t* __restrict__ head) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t p = in[i] >> shift;
        out[i] = p;
        head[i] = (i == 0 || (in[i - 1] >> shift) != p) ? 1u : 0u;
    }
}

// pre-order key of an internal node of level l (prefix of l-1 digits)
__global__ void k_order_keys(const uint64_t* __restrict__ prefix, uint64_t n, uint32_t digits, uint32_t base,
                             uint64_t* __restrict__ okey, uint32_t* __restrict__ oval) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t p = prefix[i];
        uint64_t k = 0;
        for (uint32_t j = 0; j < digits; j++) {
            const uint32_t d = uint32_t(p >> (3u * (digits - 1u - j))) & 7u;
            const uint32_t v = j == 0 ? d + 1u : 8u - d;
            k |= uint64_t(v) << (60u - 4u * j);
        }
        okey[i] = k;
        oval[i] = base + uint32_t(i);
    }
}

__global__ void k_scatter_rank(const uint32_t* __restrict__ sorted_val, uint64_t n, uint32_t* __restrict__ block) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
        block[sorted_val[i]] = 9u + 8u * uint32_t(i);
}

// words of the nodes of one level: node i's word goes to its parent's block
// (or slot 1 + digit under the root) + its last digit.  parent_of is
// 1-based, so parent_block points one element before the level's blocks.
__global__ void k_level_words(const uint64_t* __restrict__ prefix, uint64_t n, const uint32_t* __restrict__ parent_of,
                              const uint32_t* __restrict__ parent_block, const uint32_t* __restrict__ my_block,
                              const uint32_t* __restrict__ count, const uint32_t* __restrict__ material,
                              uint32_t* __restrict__ words) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t d = uint32_t(prefix[i]) & 7u;
        const uint32_t slot = (parent_block ? parent_block[parent_of[i]] : 1u) + d;
        words[slot] = my_block ? (1u | ((count[i] & 7u) << 1) | (my_block[i] << 4)) : ((material[i] & 0x7Fu) << 1);
    }
}

__global__ void k_root_word(uint32_t n_root_children, uint32_t* __restrict__ words) {
    words[0] = 1u | ((n_root_children & 7u) << 1) | (1u << 4);
}

__global__ void k_gather_material(const uint32_t* __restrict__ xyzm, const uint32_t* __restrict__ idx, uint64_t n,
                                  uint32_t* __restrict__ mat) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
        mat[i] = xyzm[4 * uint64_t(idx[i]) + 3];
}

}  // namespace build
}  // namespace ve
