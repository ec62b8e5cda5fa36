// nrc.cuh — learned radiance cache: multi-resolution hash-grid encoding and a
// 4 x 64 ReLU MLP, inference and training on the tcgen05 tensor cores.
//
// Network.  Input row (64 bf16 columns): 16 levels x 2 hash-grid features of
// the voxel centre (columns 0-31), the octahedral shading normal (32-33), the
// octahedral direction toward the previous path vertex (34-35), a constant 1
// (36), zeros (37-63).  Four hidden layers of 64 ReLU units, no biases (the
// constant input column plays that role for the first layer), a linear
// 3-channel output (layer 5 stored as 16 rows, rows 3-15 zero).  Weights are
// bf16 in the tensor-core tile layout of tc.cuh, accumulation is f32 in
// tensor memory, master weights and Adam moments are f32.
//
// Hash grid (the multiresolution hash encoding of Muller et al. 2022): level
// l has resolution floor(base * b^l) with b = (max/base)^(1/(levels-1));
// levels whose (res+1)^3 vertices fit the table are indexed densely, the
// others by (x * 1) ^ (y * 2654435761) ^ (z * 805459861) mod T.  Features are
// fp16 pairs, trilinearly interpolated in f32.
//
// Loss: relative L2, sum_c (y_c - t_c)^2 / (y_c^2 + 0.01) with y treated as a
// constant in the denominator, averaged over samples and channels.
//
// Validation: every training sample is evaluated before the step that trains
// on it; per cell of 8^3 voxels the running means of those targets and
// predictions are kept, and their relative squared difference is the cell's
// validation error (the bias of the network there, with the single-path noise
// of the targets averaged out).
//
// Kernel structure: one CTA of 128 threads per 128-row tile (thread t owns
// row t), persistent over tiles.  One thread issues the tcgen05.mma chain of a
// layer and commits it to an mbarrier; all threads wait, read their row from
// tensor memory (tcgen05.ld), apply ReLU (or its derivative) and write the
// next bf16 operand tile to shared memory.  Training keeps the five input
// tiles H0..H4 of the forward pass in shared memory and runs the backward
// pass in the same CTA: dW_l += dZ_l^T H_l accumulates per CTA in tensor
// memory across tiles (M = 64 accumulators) and is added to global f32
// gradients once per CTA; dX of the hash features is scattered into the
// table gradients with f32 atomics.
#pragma once
#include <cuda_fp16.h>

#include "tc.cuh"

namespace ve {
namespace nrc {

constexpr uint32_t kLevels = 16;
constexpr uint32_t kWidth = 64;
constexpr uint32_t kLayers = 5;
constexpr uint32_t kRows = 128;
constexpr uint32_t kTileBytes = kRows * kWidth * 2;       // 16 KB
constexpr uint32_t kWBytes = kWidth * kWidth * 2;         // 8 KB per layer image
constexpr uint32_t kWImage = kLayers * kWBytes;           // 40 KB
constexpr uint32_t kWParams = kLayers * kWidth * kWidth;  // f32 master weights (layer 5 rows >= 3 are zero)
constexpr uint32_t kOutRows = 3;
constexpr uint32_t kInferGroups = 2;  // warpgroups (independent tile streams) per inference CTA
constexpr uint32_t kSmemInfer = kWImage + kInferGroups * kTileBytes;
constexpr uint32_t kSmemTrain = kWImage + 6 * kTileBytes;
constexpr uint32_t kTmemInfer = 64 * kInferGroups;
constexpr uint32_t kTmemTrain = 512;
constexpr long long kWaitCycles = 2000000000ll;  // ~1 s at 1.9 GHz

// Inputs of one query / sample (32 B).
struct QRec {
    float px, py, pz;  // voxel centre / scene extent, in [0,1)^3
    uint32_t path;     // path id (queries); unused for samples
    float nx, ny;      // octahedral shading normal
    float vx, vy;      // octahedral direction toward the previous vertex
};

// Training target of one sample (48 B).  The shade pass fills tp / s1 at the
// recorded vertex and the target when the path ends.
struct TRec {
    float tr, tg, tb;  // target radiance leaving the vertex
    uint32_t valid;
    float t0, t1, t2;  // path throughput arriving at the vertex
    uint32_t cell;     // validation-error cell (0xFFFFFFFF: none)
    float s0, s1, s2;  // radiance the path had gathered before the vertex
    uint32_t pad;
};

struct Grid {
    uint32_t res[kLevels];
    uint32_t dense_mask;
    uint32_t log2T;
};

struct Args {
    const QRec* q;
    const TRec* tr;            // training only
    const uint32_t* count;     // device row count (nullptr: n)
    uint32_t n;                // capacity / row count
    const uint32_t* table;     // fp16 feature pairs, levels x T
    const uint4* wimg;         // bf16 weight image (kWImage bytes)
    Grid grid;
    float4* out;               // inference: prediction per row
    float* wgrad;              // training: f32 [5][64][64]
    float* tgrad;              // training: f32 [levels][T][2]
    float* loss;               // training: sum of per-sample losses
    float4* val;               // training: per cell {mean target rgb, samples}, {mean prediction rgb, -}
    uint32_t val_mask;
    float inv_norm;            // 1 / (3 * rows)
    uint32_t* status;          // bit 0: a wait timed out
    uint32_t* nvalid;          // training: samples with a target
};

__device__ __forceinline__ void level_corners(const Grid& g, uint32_t l, float px, float py, float pz,
                                              uint32_t (&idx)[8], float (&w)[8]) {
    const uint32_t R = g.res[l];
    const float s = float(R);
    const float x = px * s, y = py * s, z = pz * s;
    const float fx0 = floorf(x), fy0 = floorf(y), fz0 = floorf(z);
    const uint32_t ix = min(uint32_t(fmaxf(fx0, 0.0f)), R - 1u);
    const uint32_t iy = min(uint32_t(fmaxf(fy0, 0.0f)), R - 1u);
    const uint32_t iz = min(uint32_t(fmaxf(fz0, 0.0f)), R - 1u);
    const float fx = x - float(ix), fy = y - float(iy), fz = z - float(iz);
    const uint32_t T = 1u << g.log2T;
    const bool dense = (g.dense_mask >> l) & 1u;
    const uint32_t R1 = R + 1u;
#pragma unroll
    for (uint32_t c = 0; c < 8; c++) {
        const uint32_t cx = ix + (c & 1u), cy = iy + ((c >> 1) & 1u), cz = iz + ((c >> 2) & 1u);
        idx[c] = dense ? (cx + R1 * (cy + R1 * cz)) : ((cx ^ (cy * 2654435761u) ^ (cz * 805459861u)) & (T - 1u));
        const float wx = (c & 1u) ? fx : 1.0f - fx;
        const float wy = (c & 2u) ? fy : 1.0f - fy;
        const float wz = (c & 4u) ? fz : 1.0f - fz;
        w[c] = (wx * wy) * wz;
    }
}

// Input row of a record as 32 packed bf16 pairs.
__device__ __forceinline__ void encode_row(const Args& a, const QRec& r, bool valid, uint32_t (&row)[32]) {
#pragma unroll
    for (int i = 0; i < 32; i++) row[i] = 0u;
    if (!valid) return;
    const uint32_t T = 1u << a.grid.log2T;
    // two levels per round: 16 independent gathers in flight per thread
#pragma unroll 1
    for (uint32_t l = 0; l < kLevels; l += 2) {
        uint32_t idx[2][8], h[2][8];
        float w[2][8];
        level_corners(a.grid, l, r.px, r.py, r.pz, idx[0], w[0]);
        level_corners(a.grid, l + 1u, r.px, r.py, r.pz, idx[1], w[1]);
#pragma unroll
        for (int k = 0; k < 2; k++)
#pragma unroll
            for (int c = 0; c < 8; c++) h[k][c] = __ldg(a.table + size_t(l + k) * T + idx[k][c]);
#pragma unroll
        for (int k = 0; k < 2; k++) {
            float f0 = 0.0f, f1 = 0.0f;
#pragma unroll
            for (int c = 0; c < 8; c++) {
                const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&h[k][c]));
                f0 += w[k][c] * f.x;
                f1 += w[k][c] * f.y;
            }
            row[l + k] = tc::pack_bf16(f0, f1);
        }
    }
    row[16] = tc::pack_bf16(r.nx, r.ny);
    row[17] = tc::pack_bf16(r.vx, r.vy);
    row[18] = tc::pack_bf16(1.0f, 0.0f);
}

__device__ __forceinline__ void store_row(uint8_t* tile, uint32_t t, const uint32_t (&row)[32]) {
#pragma unroll
    for (uint32_t j = 0; j < 8; j++)
        *reinterpret_cast<uint4*>(tile + tc::tile_off(t, 8u * j)) =
            make_uint4(row[4 * j], row[4 * j + 1], row[4 * j + 2], row[4 * j + 3]);
}

// Issues layer `l` of the forward pass: D(128 x N) = A(128 x 64) W_l^T.
__device__ __forceinline__ void issue_forward(uint32_t t_scr, const uint8_t* A, const uint8_t* W, uint32_t N) {
    const uint32_t a0 = tc::smem_u32(A), w0 = tc::smem_u32(W);
    const uint32_t id = tc::idesc_bf16(128u, N, 0u, 0u);
#pragma unroll
    for (uint32_t kk = 0; kk < 4; kk++) tc::mma_bf16(t_scr, tc::kmajor(a0 + 256u * kk), tc::kmajor(w0 + 256u * kk), id, kk);
}

template <bool TRAIN>
__global__ void __launch_bounds__(128, TRAIN ? 1 : 4) k_nrc_mlp(Args a) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ uint64_t mbar;
    __shared__ uint32_t tmem_base;
    uint8_t* sw = smem;
    uint8_t* sh = smem + kWImage;
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
    constexpr uint32_t kCols = TRAIN ? kTmemTrain : kTmemInfer;

    for (uint32_t i = tid; i < kWImage / 16u; i += blockDim.x)
        reinterpret_cast<uint4*>(sw)[i] = __ldg(a.wimg + i);
    if (warp == 0) {
        tc::tmem_alloc(&tmem_base, kCols);
        tc::tmem_relinquish();
    }
    if (tid == 0) tc::mbar_init(&mbar, 1u);
    tc::fence_async_smem();
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = tmem_base;
    const uint32_t t_scr = tmem;
    const uint32_t lane_sel = (warp * 32u) << 16;
    uint32_t phase = 0;
    bool timed_out = false;
    bool any = false;
    float loss_sum = 0.0f;
    uint32_t n_valid = 0;
    const uint32_t n = a.count ? min(*a.count, a.n) : a.n;
    const uint32_t tiles = (n + kRows - 1u) / kRows;
    const uint32_t T = 1u << a.grid.log2T;

    for (uint32_t tile = blockIdx.x; tile < tiles && !timed_out; tile += gridDim.x) {
        const uint32_t row = tile * kRows + tid;
        QRec r{};
        TRec tr{};
        bool valid = row < n;
        if (valid) r = a.q[row];
        if (TRAIN && valid) {
            tr = a.tr[row];
            valid = tr.valid != 0u;
        }
        {
            uint32_t x[32];
            encode_row(a, r, valid, x);
            store_row(sh, tid, x);
        }
        tc::fence_async_smem();
        tc::fence_before();
        __syncthreads();
        float y[3] = {0.0f, 0.0f, 0.0f};
        // ---- forward ----
        for (uint32_t l = 0; l < kLayers; l++) {
            const uint8_t* A = TRAIN ? sh + l * kTileBytes : sh;
            if (tid == 0) {
                tc::fence_after();
                issue_forward(t_scr, A, sw + l * kWBytes, l + 1u < kLayers ? 64u : 16u);
                tc::commit(&mbar);
            }
            if (!tc::mbar_wait(&mbar, phase, kWaitCycles)) {
                timed_out = true;
                break;
            }
            phase ^= 1u;
            tc::fence_after();
            if (l + 1u < kLayers) {
                uint8_t* dst = TRAIN ? sh + (l + 1u) * kTileBytes : sh;
#pragma unroll
                for (uint32_t half = 0; half < 2; half++) {
                    uint32_t v[32];
                    tc::tmem_ld32(t_scr + lane_sel + 32u * half, v);
                    tc::tmem_wait_ld();
                    uint32_t pk[16];
#pragma unroll
                    for (int j = 0; j < 16; j++)
                        pk[j] = tc::pack_bf16(fmaxf(__uint_as_float(v[2 * j]), 0.0f),
                                              fmaxf(__uint_as_float(v[2 * j + 1]), 0.0f));
#pragma unroll
                    for (uint32_t c = 0; c < 4; c++)
                        *reinterpret_cast<uint4*>(dst + tc::tile_off(tid, 32u * half + 8u * c)) =
                            make_uint4(pk[4 * c], pk[4 * c + 1], pk[4 * c + 2], pk[4 * c + 3]);
                }
                tc::fence_async_smem();
                tc::fence_before();
                __syncthreads();
            } else {
                uint32_t v[32];
                tc::tmem_ld32(t_scr + lane_sel, v);
                tc::tmem_wait_ld();
                y[0] = __uint_as_float(v[0]);
                y[1] = __uint_as_float(v[1]);
                y[2] = __uint_as_float(v[2]);
            }
        }
        if (timed_out) break;
        if (!TRAIN) {
            if (row < n) a.out[row] = make_float4(y[0], y[1], y[2], 0.0f);
            tc::fence_before();
            __syncthreads();
            continue;
        }
        // ---- loss and output gradient ----
        {
            const float tv[3] = {tr.tr, tr.tg, tr.tb};
            float d[3];
            float e = 0.0f;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const float den = y[c] * y[c] + 0.01f;
                const float diff = y[c] - tv[c];
                e += (diff * diff) / den;
                d[c] = valid ? (2.0f * diff / den) * a.inv_norm : 0.0f;
            }
            if (valid) {
                loss_sum += e;
                n_valid++;
                if (a.val && tr.cell != 0xFFFFFFFFu) {
                    // validation statistics of the cell: running means of the
                    // targets and of the (not yet updated) network's predictions
                    float4* cs = a.val + 2u * (tr.cell & a.val_mask);
                    float4 et = cs[0], ey = cs[1];
                    const float cnt = et.w + 1.0f;
                    const float wgt = fmaxf(1.0f / cnt, 0.05f);
                    et = make_float4(et.x + wgt * (tv[0] - et.x), et.y + wgt * (tv[1] - et.y), et.z + wgt * (tv[2] - et.z), cnt);
                    ey = make_float4(ey.x + wgt * (y[0] - ey.x), ey.y + wgt * (y[1] - ey.y), ey.z + wgt * (y[2] - ey.z), 0.0f);
                    cs[0] = et;
                    cs[1] = ey;
                }
            }
            uint32_t g[32];
#pragma unroll
            for (int i = 0; i < 32; i++) g[i] = 0u;
            g[0] = tc::pack_bf16(d[0], d[1]);
            g[1] = tc::pack_bf16(d[2], 0.0f);
            store_row(sh + 5u * kTileBytes, tid, g);
        }
        tc::fence_async_smem();
        tc::fence_before();
        __syncthreads();
        // ---- backward ----
        uint8_t* G = sh + 5u * kTileBytes;
        for (int l = int(kLayers) - 1; l >= 0; l--) {
            const uint8_t* Hin = sh + uint32_t(l) * kTileBytes;
            if (tid == 0) {
                tc::fence_after();
                const uint32_t g0 = tc::smem_u32(G), h0 = tc::smem_u32(Hin), w0 = tc::smem_u32(sw + uint32_t(l) * kWBytes);
                const uint32_t t_dw = tmem + 64u + 64u * uint32_t(l);
                const uint32_t id_w = tc::idesc_bf16(64u, 64u, 1u, 1u);
#pragma unroll
                for (uint32_t kk = 0; kk < 8; kk++)
                    tc::mma_bf16(t_dw, tc::mnmajor(g0 + 2048u * kk), tc::mnmajor(h0 + 2048u * kk), id_w,
                                 (any || kk > 0u) ? 1u : 0u);
                const uint32_t kout = l == int(kLayers) - 1 ? 1u : 4u;  // K = 16 or 64 output units
                const uint32_t id_d = tc::idesc_bf16(128u, 64u, 0u, 1u);
                for (uint32_t kk = 0; kk < kout; kk++)
                    tc::mma_bf16(t_scr, tc::kmajor(g0 + 256u * kk), tc::mnmajor(w0 + 2048u * kk), id_d, kk);
                tc::commit(&mbar);
            }
            if (!tc::mbar_wait(&mbar, phase, kWaitCycles)) {
                timed_out = true;
                break;
            }
            phase ^= 1u;
            tc::fence_after();
            if (l > 0) {
                // dZ_{l-1} = dH_l * [H_l > 0]
#pragma unroll
                for (uint32_t half = 0; half < 2; half++) {
                    uint32_t v[32];
                    tc::tmem_ld32(t_scr + lane_sel + 32u * half, v);
                    tc::tmem_wait_ld();
                    uint32_t pk[16];
#pragma unroll
                    for (uint32_t c = 0; c < 4; c++) {
                        const uint4 hv = *reinterpret_cast<const uint4*>(Hin + tc::tile_off(tid, 32u * half + 8u * c));
                        const uint32_t hw[4] = {hv.x, hv.y, hv.z, hv.w};
#pragma unroll
                        for (int j = 0; j < 4; j++) {
                            const float g_lo = tc::bf16_lo(hw[j]) > 0.0f ? __uint_as_float(v[8 * c + 2 * j]) : 0.0f;
                            const float g_hi = tc::bf16_hi(hw[j]) > 0.0f ? __uint_as_float(v[8 * c + 2 * j + 1]) : 0.0f;
                            pk[4 * c + j] = tc::pack_bf16(g_lo, g_hi);
                        }
                    }
#pragma unroll
                    for (uint32_t c = 0; c < 4; c++)
                        *reinterpret_cast<uint4*>(G + tc::tile_off(tid, 32u * half + 8u * c)) =
                            make_uint4(pk[4 * c], pk[4 * c + 1], pk[4 * c + 2], pk[4 * c + 3]);
                }
                tc::fence_async_smem();
                tc::fence_before();
                __syncthreads();
            } else {
                // dX of the hash features (columns 0-31) -> table gradients
                uint32_t v[32];
                tc::tmem_ld32(t_scr + lane_sel, v);
                tc::tmem_wait_ld();
                if (valid) {
#pragma unroll 1
                    for (uint32_t lv = 0; lv < kLevels; lv++) {
                        uint32_t idx[8];
                        float w[8];
                        level_corners(a.grid, lv, r.px, r.py, r.pz, idx, w);
                        const float g0 = __uint_as_float(v[2 * lv]), g1 = __uint_as_float(v[2 * lv + 1]);
#pragma unroll
                        for (int c = 0; c < 8; c++) {
                            float* dst = a.tgrad + 2ull * (size_t(lv) * T + idx[c]);
                            atomicAdd(reinterpret_cast<float2*>(dst), make_float2(w[c] * g0, w[c] * g1));
                        }
                    }
                }
                tc::fence_before();
                __syncthreads();
            }
        }
        any = true;
    }
    if (timed_out) {
        if (tid == 0) atomicOr(a.status, 1u);
    } else if (TRAIN) {
        tc::fence_before();
        __syncthreads();
        tc::fence_after();
        if (any) {
            // M = 64 accumulators: row o lives in lane (o % 16) + 32 * (o / 16)
            for (uint32_t l = 0; l < kLayers; l++) {
                const uint32_t rows = l + 1u < kLayers ? 64u : kOutRows;
                const uint32_t o = 16u * warp + lane;
#pragma unroll
                for (uint32_t half = 0; half < 2; half++) {
                    uint32_t v[32];
                    tc::tmem_ld32(tmem + 64u + 64u * l + lane_sel + 32u * half, v);
                    tc::tmem_wait_ld();
                    if (lane < 16u && o < rows) {
                        float* dst = a.wgrad + size_t(l) * kWidth * kWidth + size_t(o) * kWidth + 32u * half;
#pragma unroll
                        for (int j = 0; j < 32; j++) atomicAdd(dst + j, __uint_as_float(v[j]));
                    }
                }
            }
        }
        float s = loss_sum;
        uint32_t nvs = n_valid;
        for (int off = 16; off > 0; off >>= 1) {
            s += __shfl_xor_sync(0xffffffffu, s, off);
            nvs += __shfl_xor_sync(0xffffffffu, nvs, off);
        }
        if (lane == 0 && s != 0.0f) atomicAdd(a.loss, s);
        if (lane == 0 && nvs) atomicAdd(a.nvalid, nvs);
    }
    tc::fence_before();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, kCols);
}

__device__ __forceinline__ void group_sync(uint32_t g) {
    asm volatile("bar.sync %0, 128;" ::"r"(1u + g) : "memory");
}

// Inference, step 1: the input rows of the queries, in the operand-tile
// image (tile t at X + 16 KB * t, row r at tile_off(r, .)).  The hash-grid
// gathers are latency-bound; this kernel runs at full occupancy so enough of
// them are in flight, and the MLP kernel then copies finished tiles.
// `pre(row, r)` may stage per-row data for the MLP kernel's epilogue (the
// frame form gathers the query path's state here, so the epilogue reads it
// coalesced).
struct NoStage {
    __device__ __forceinline__ void operator()(uint32_t, const QRec&) const {}
};

template <class Pre>
__global__ void __launch_bounds__(256, 4) k_nrc_encode(Args a, uint8_t* __restrict__ X, Pre pre) {
    const uint32_t n = a.count ? min(*a.count, a.n) : a.n;
    const uint32_t T = 1u << a.grid.log2T;
    for (uint32_t row = blockIdx.x * blockDim.x + threadIdx.x; row < n; row += gridDim.x * blockDim.x) {
        const QRec r = a.q[row];
        pre(row, r);
        uint8_t* tile = X + size_t(row / kRows) * kTileBytes;
        const uint32_t t = row % kRows;
        // columns 8j..8j+7 = levels 4j..4j+3, streamed out one 16-byte chunk at a time
#pragma unroll 1
        for (uint32_t j = 0; j < 4; j++) {
            uint32_t pk[4];
#pragma unroll
            for (uint32_t k = 0; k < 4; k += 2) {
                uint32_t idx[2][8], h[2][8];
                float w[2][8];
                level_corners(a.grid, 4u * j + k, r.px, r.py, r.pz, idx[0], w[0]);
                level_corners(a.grid, 4u * j + k + 1u, r.px, r.py, r.pz, idx[1], w[1]);
#pragma unroll
                for (int e = 0; e < 2; e++)
#pragma unroll
                    for (int c = 0; c < 8; c++) h[e][c] = __ldg(a.table + size_t(4u * j + k + e) * T + idx[e][c]);
#pragma unroll
                for (int e = 0; e < 2; e++) {
                    float f0 = 0.0f, f1 = 0.0f;
#pragma unroll
                    for (int c = 0; c < 8; c++) {
                        const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&h[e][c]));
                        f0 += w[e][c] * f.x;
                        f1 += w[e][c] * f.y;
                    }
                    pk[k + e] = tc::pack_bf16(f0, f1);
                }
            }
            *reinterpret_cast<uint4*>(tile + tc::tile_off(t, 8u * j)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
        }
        *reinterpret_cast<uint4*>(tile + tc::tile_off(t, 32u)) =
            make_uint4(tc::pack_bf16(r.nx, r.ny), tc::pack_bf16(r.vx, r.vy), tc::pack_bf16(1.0f, 0.0f), 0u);
        for (uint32_t j = 5; j < 8; j++)
            *reinterpret_cast<uint4*>(tile + tc::tile_off(t, 8u * j)) = make_uint4(0u, 0u, 0u, 0u);
    }
}

// Output of one inference row: the host-API form stores the prediction.
struct StoreOut {
    float4* out;
    __device__ __forceinline__ void operator()(uint8_t*, uint32_t row, bool valid, const float (&y)[3]) const {
        if (valid) out[row] = make_float4(y[0], y[1], y[2], 0.0f);
    }
};

// Inference, step 2: two warpgroups per CTA run independent tile streams,
// each with its own operand tile, tensor-memory columns (M = 128
// accumulator, lanes 0-127) and mbarrier, so one group's tile copy and
// epilogue overlap the other's tensor-core work; three CTAs per SM (shared
// memory, and 384 of the 512 tensor-memory columns).  `epi(scratch, row,
// valid, y)` is called by all 128 threads of a group with the row's
// prediction; `scratch` is 4 KB of shared memory free during the call.
template <class Epi>
__global__ void __launch_bounds__(256, 3) k_nrc_infer(Args a, const uint8_t* __restrict__ X, Epi epi) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ uint64_t mbar[kInferGroups];
    __shared__ uint32_t tmem_base;
    uint8_t* sw = smem;
    const uint32_t tid = threadIdx.x, g = tid >> 7, t = tid & 127u, warp = tid >> 5;
    uint8_t* sh = smem + kWImage + g * kTileBytes;

    for (uint32_t i = tid; i < kWImage / 16u; i += blockDim.x)
        reinterpret_cast<uint4*>(sw)[i] = __ldg(a.wimg + i);
    if (warp == 0) {
        tc::tmem_alloc(&tmem_base, kTmemInfer);
        tc::tmem_relinquish();
    }
    if (tid == 0)
        for (uint32_t k = 0; k < kInferGroups; k++) tc::mbar_init(&mbar[k], 1u);
    tc::fence_async_smem();
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t t_scr = tmem_base + 64u * g;
    const uint32_t lane_sel = ((warp & 3u) * 32u) << 16;  // the warp's quarter of the lanes
    uint32_t phase = 0;
    bool timed_out = false;
    const uint32_t n = a.count ? min(*a.count, a.n) : a.n;
    const uint32_t tiles = (n + kRows - 1u) / kRows;
    for (uint32_t tile = blockIdx.x * kInferGroups + g; tile < tiles && !timed_out;
         tile += gridDim.x * kInferGroups) {
        const uint32_t row = tile * kRows + t;
        const bool valid = row < n;
        {   // the tile image, 16 KB contiguous: coalesced 16-byte copies
            const uint4* src = reinterpret_cast<const uint4*>(X + size_t(tile) * kTileBytes);
#pragma unroll
            for (uint32_t j = 0; j < kTileBytes / 16u / 128u; j++)
                reinterpret_cast<uint4*>(sh)[j * 128u + t] = __ldg(src + j * 128u + t);
        }
        tc::fence_async_smem();
        tc::fence_before();
        group_sync(g);
        float y[3] = {0.0f, 0.0f, 0.0f};
        for (uint32_t l = 0; l < kLayers; l++) {
            if (t == 0) {
                tc::fence_after();
                issue_forward(t_scr, sh, sw + l * kWBytes, l + 1u < kLayers ? 64u : 16u);
                tc::commit(&mbar[g]);
            }
            if (!tc::mbar_wait(&mbar[g], phase, kWaitCycles)) {
                timed_out = true;
                break;
            }
            phase ^= 1u;
            tc::fence_after();
            if (l + 1u < kLayers) {
#pragma unroll
                for (uint32_t half = 0; half < 2; half++) {
                    uint32_t v[32];
                    tc::tmem_ld32(t_scr + lane_sel + 32u * half, v);
                    tc::tmem_wait_ld();
                    uint32_t pk[16];
#pragma unroll
                    for (int j = 0; j < 16; j++)
                        pk[j] = tc::pack_bf16(fmaxf(__uint_as_float(v[2 * j]), 0.0f),
                                              fmaxf(__uint_as_float(v[2 * j + 1]), 0.0f));
#pragma unroll
                    for (uint32_t c = 0; c < 4; c++)
                        *reinterpret_cast<uint4*>(sh + tc::tile_off(t, 32u * half + 8u * c)) =
                            make_uint4(pk[4 * c], pk[4 * c + 1], pk[4 * c + 2], pk[4 * c + 3]);
                }
                tc::fence_async_smem();
                tc::fence_before();
                group_sync(g);
            } else {
                uint32_t v[32];
                tc::tmem_ld32(t_scr + lane_sel, v);
                tc::tmem_wait_ld();
                y[0] = __uint_as_float(v[0]);
                y[1] = __uint_as_float(v[1]);
                y[2] = __uint_as_float(v[2]);
            }
        }
        if (timed_out) break;
        epi(sh, row, valid, y);  // the last layer's operands are consumed: sh is scratch
        tc::fence_before();
        group_sync(g);
    }
    if (timed_out && t == 0) atomicOr(a.status, 1u);
    tc::fence_before();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem_base, kTmemInfer);
}

// ---------------------------------------------------------------------------
// Adam (Kingma & Ba 2015).  The step's bias corrections live in device memory
// (written by k_nrc_step) so that the update can be replayed from a graph.
struct AdamState {
    uint32_t step;
    float bc1, bc2;  // 1 - beta1^t, 1 - beta2^t
    float pad;
};

__global__ void k_nrc_step(AdamState* s, float b1, float b2) {
    const uint32_t t = s->step + 1u;
    s->step = t;
    s->bc1 = 1.0f - powf(b1, float(t));
    s->bc2 = 1.0f - powf(b2, float(t));
}

struct AdamArgs {
    float lr, b1, b2, eps;
    const AdamState* st;
};

__device__ __forceinline__ float adam_update(float& p, float& m, float& v, float g, const AdamArgs& a, float bc1,
                                             float bc2) {
    m = a.b1 * m + (1.0f - a.b1) * g;
    v = a.b2 * v + (1.0f - a.b2) * (g * g);
    const float mh = m / bc1, vh = v / bc2;
    p -= a.lr * mh / (sqrtf(vh) + a.eps);
    return p;
}

// Weights: updates the f32 masters, clears the gradients and rewrites the
// bf16 tensor-core image.  Layer-5 rows >= 3 stay zero.
__global__ void k_nrc_adam_weights(float* w, float* m, float* v, float* g, uint8_t* img, AdamArgs a) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kWParams) return;
    const uint32_t l = i / (kWidth * kWidth), o = (i / kWidth) % kWidth, c = i % kWidth;
    float p = w[i];
    if (l + 1u == kLayers && o >= kOutRows) {
        p = 0.0f;
    } else {
        float mm = m[i], vv = v[i];
        adam_update(p, mm, vv, g[i], a, a.st->bc1, a.st->bc2);
        m[i] = mm;
        v[i] = vv;
    }
    w[i] = p;
    g[i] = 0.0f;
    const uint16_t b = uint16_t(tc::pack_bf16(p, 0.0f) & 0xFFFFu);
    *reinterpret_cast<uint16_t*>(img + size_t(l) * kWBytes + tc::tile_off(o, c)) = b;
}

// Hash table: f32 master pairs -> fp16 pairs.  Entries whose gradient is zero
// still decay their moments (dense Adam).
__global__ void k_nrc_adam_table(float2* p, float2* m, float2* v, float2* g, uint32_t* h, size_t n, AdamArgs a) {
    const float bc1 = a.st->bc1, bc2 = a.st->bc2;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        float2 pp = p[i], mm = m[i], vv = v[i];
        const float2 gg = g[i];
        adam_update(pp.x, mm.x, vv.x, gg.x, a, bc1, bc2);
        adam_update(pp.y, mm.y, vv.y, gg.y, a, bc1, bc2);
        p[i] = pp;
        m[i] = mm;
        v[i] = vv;
        g[i] = make_float2(0.0f, 0.0f);
        const __half2 hv = __floats2half2_rn(pp.x, pp.y);
        h[i] = *reinterpret_cast<const uint32_t*>(&hv);
    }
}

// f32 parameter images -> device formats (set_params).
__global__ void k_nrc_weights_image(const float* w, uint8_t* img) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kWParams) return;
    const uint32_t l = i / (kWidth * kWidth), o = (i / kWidth) % kWidth, c = i % kWidth;
    const float p = (l + 1u == kLayers && o >= kOutRows) ? 0.0f : w[i];
    *reinterpret_cast<uint16_t*>(img + size_t(l) * kWBytes + tc::tile_off(o, c)) =
        uint16_t(tc::pack_bf16(p, 0.0f) & 0xFFFFu);
}
__global__ void k_nrc_table_half(const float2* p, uint32_t* h, size_t n) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const __half2 hv = __floats2half2_rn(p[i].x, p[i].y);
        h[i] = *reinterpret_cast<const uint32_t*>(&hv);
    }
}

}  // namespace nrc
}  // namespace ve
