// Fused inference of the surrogate ensemble: one persistent kernel runs every member's five layers
// (64 -> 512 -> 512 -> 512 -> 512 -> 128, GELU between) for tiles of 128 queries and applies the
// disagreement gate, without writing an activation to global memory.
//
// Per CTA (one per SM, 18 warps):
//   warp 0, one lane   producer: streams the members' weights, pre-packed in the order they are
//                      consumed (tmc_b200_nn_pack), through three 32 KB shared-memory stages with
//                      bulk copies (cp.async.bulk, completion counted on the stage's mbarrier);
//   warp 1, one lane   tensor-core issuer: for each layer, tcgen05.mma of the 128 x K activation
//                      tile (shared memory) by each weight tile into the TMEM accumulator (128 lanes x
//                      up to 512 FP32 columns; N is issued in halves of 256), committing each stage
//                      back to the producer and the finished layer to the epilogue;
//   warps 2-17         epilogue: read the accumulator with tcgen05.ld (warp w owns TMEM lanes
//                      32 (w % 4) .. + 31, i.e. query rows, and a quarter of the columns), add the bias,
//                      apply GELU, and write the BF16 activations back into the activation tile in
//                      the 128-byte-swizzled K-major layout the next layer's MMA reads; after the
//                      output layer they de-normalise, accumulate the members' mean, sum each
//                      member's R_d on the grid (sum of 10^y * annulus area) and finally write the
//                      mean outputs, the mean R_d, the spread (sample standard deviation over the
//                      mean) and the route flag. They also encode the raw features (z-score, BF16,
//                      zero padding to 64) into the activation tile before each member.
//
// Hand-offs are mbarriers: full[s] / empty[s] between producer and issuer, acc_full (issuer ->
// epilogue, one phase per layer), act_ready (epilogue -> issuer, 512 arrivals per phase: the
// activation tile is written and the accumulator read) and rdx (the warps holding R_d bins 32-63
// hand their partial sums to those holding bins 0-31, once per member). Every wait is bounded: a
// wait that gives up raises the device status word and a shared abort flag, every role leaves its
// loop (warp-uniformly), the producer waits (bounded) for its copies in flight, the issuer for its
// MMAs in flight, and the CTA frees its TMEM and returns.
#pragma once

#include <cuda_bf16.h>

#include "umma.cuh"

namespace tmc {

constexpr int kInferThreads = 576;        // 18 warps
constexpr int kInferStages = 3;
constexpr int kInferStageBytes = 32768;   // 256 rows x 64 bf16
constexpr int kInferChunkBytes = 16384;   // 128 rows x 64 bf16
constexpr int kInferLayers = 5;
constexpr int kInferHidden = 512, kInferIn = 64, kInferOut = 128;
constexpr int kInferBiasPerMember = 4 * kInferHidden + kInferOut;  // 2176
// tiles per member in stream order: layer 0 (2 halves x 1 K chunk), layers 1-3 (2 x 8), layer 4 (1 x 8)
constexpr int kInferTilesPerMember = 2 + 3 * 16 + 8;
constexpr int kInferBigTiles = 2 + 3 * 16;  // 32 KB each; the last 8 are 16 KB
constexpr uint32_t kInferMemberBytes = kInferBigTiles * 32768u + 8u * 16384u;  // 1,769,472
constexpr int kInferMaxMembers = 8;
constexpr uint32_t kInferWaitLimit = 1u << 24;

struct InferSmem {
    static constexpr int a = 0;                                          // 8 chunks x 16 KB
    static constexpr int stages = a + 8 * kInferChunkBytes;              // 131072
    static constexpr int rdx = stages + kInferStages * kInferStageBytes; // 229376: 2 x 128 floats
    static constexpr int bars = rdx + 2 * 128 * 4;                       // 230400: 10 mbarriers
    static constexpr int tmem_slot = bars + 10 * 8;
    static constexpr int abort_flag = tmem_slot + 4;
    static constexpr int bytes = abort_flag + 4 + 1024;  // + alignment slack
};

struct InferParams {
    const unsigned char *packed;  // members x kInferMemberBytes
    const float *bias;            // members x 2176: b0[512] b1[512] b2[512] b3[512] b4[128]
    const float *feats;           // n x n_feat raw features
    const float *x_mean, *x_std;  // n_feat
    const float *y_mean, *y_std;  // n_out
    const float *areas;           // nbins
    float *out;                   // n x n_out, optional
    float *rd_mean, *spread;      // n, optional
    unsigned char *route;         // n, optional
    int n, n_feat, n_out, nbins, members;
    float threshold;
    int *status;
};

// ------------------------------------------------------------------------------ weight packing
// Packed tile (rows x 64 bf16 of W[row0 + r][k0 + k]): byte r * 128 + ((k / 8) ^ (r % 8)) * 16 + (k % 8) * 2.
struct PackParams {
    const __nv_bfloat16 *w[kInferMaxMembers * kInferLayers];  // per member: 512x64, 512x512 x3, 128x512
    int members;
};

__global__ void pack_kernel(const __grid_constant__ PackParams P, unsigned char *__restrict__ packed) {
    const size_t units_per_member = kInferMemberBytes / 16;
    const size_t u = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (u >= units_per_member * P.members) return;
    const int m = static_cast<int>(u / units_per_member);
    uint32_t off = static_cast<uint32_t>(u % units_per_member) * 16u;  // byte offset inside the member
    // locate the tile
    int layer, half, kc;
    uint32_t in_tile;
    if (off < 2u * 32768u) {
        layer = 0;
        half = static_cast<int>(off / 32768u);
        kc = 0;
        in_tile = off % 32768u;
    } else if (off < static_cast<uint32_t>(kInferBigTiles) * 32768u) {
        const uint32_t t = (off - 2u * 32768u) / 32768u;  // 0..47
        layer = 1 + static_cast<int>(t / 16u);
        half = static_cast<int>((t % 16u) / 8u);
        kc = static_cast<int>(t % 8u);
        in_tile = (off - 2u * 32768u) % 32768u;
    } else {
        const uint32_t o = off - static_cast<uint32_t>(kInferBigTiles) * 32768u;
        layer = 4;
        half = 0;
        kc = static_cast<int>(o / 16384u);
        in_tile = o % 16384u;
    }
    const int r = static_cast<int>(in_tile / 128u);
    const int unit = static_cast<int>((in_tile % 128u) / 16u) ^ (r & 7);  // logical 8-element group
    const int K = layer == 0 ? kInferIn : kInferHidden;
    const __nv_bfloat16 *W = P.w[m * kInferLayers + layer];
    const uint4 v = *reinterpret_cast<const uint4 *>(W + static_cast<size_t>(half * 256 + r) * K + kc * 64 + unit * 8);
    *reinterpret_cast<uint4 *>(packed + static_cast<size_t>(m) * kInferMemberBytes + off) = v;
}

// ------------------------------------------------------------------------------ the fused kernel
__device__ __forceinline__ float infer_gelu(float x) { return gelu_tanh(x); }

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t *>(&h);
}

// Byte address of columns [c, c + 8) of row r in the swizzled activation tile (c a multiple of 8).
__device__ __forceinline__ unsigned char *act_unit(unsigned char *A, int r, int c) {
    return A + (c >> 6) * kInferChunkBytes + r * 128 + ((((c & 63) >> 3) ^ (r & 7)) << 4);
}

__device__ __forceinline__ bool infer_wait(uint64_t *bar, uint32_t parity, volatile int *abort_flag, int *status) {
    if (*abort_flag) return false;
    if (mbar_wait(bar, parity, kInferWaitLimit)) return true;
    *abort_flag = 1;
    atomicExch(status, 1);
    return false;
}

// Encode rows [row0, row0 + 128) of the raw features into activation chunk 0 (512 epilogue threads).
__device__ __forceinline__ void infer_encode(const InferParams &P, unsigned char *A, int row0, int et) {
    const int r = et >> 2, part = et & 3;  // 128 rows x 4 parts of 16 columns
    const int g = row0 + r;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int c0 = part * 16 + h * 8;
        float v[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int c = c0 + i;
            v[i] = (g < P.n && c < P.n_feat) ? (P.feats[static_cast<size_t>(g) * P.n_feat + c] - P.x_mean[c]) / P.x_std[c]
                                             : 0.0f;
        }
        const uint4 u = make_uint4(pack_bf16x2(v[0], v[1]), pack_bf16x2(v[2], v[3]), pack_bf16x2(v[4], v[5]),
                                   pack_bf16x2(v[6], v[7]));
        *reinterpret_cast<uint4 *>(act_unit(A, r, c0)) = u;
    }
}

__device__ __forceinline__ void epi_release(uint64_t *act_ready) {
    fence_async_smem();  // activation writes visible to the tensor core's async proxy
    tc_fence_before();   // accumulator reads ordered before the hand-off
    mbar_arrive(act_ready);
}

__global__ void __launch_bounds__(kInferThreads, 1) ensemble_infer_kernel(const __grid_constant__ InferParams P) {
    extern __shared__ unsigned char ism_raw[];
    unsigned char *base = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(ism_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    unsigned char *A = base + InferSmem::a;
    unsigned char *stages = base + InferSmem::stages;
    float *rdx = reinterpret_cast<float *>(base + InferSmem::rdx);
    uint64_t *bars = reinterpret_cast<uint64_t *>(base + InferSmem::bars);
    uint64_t *full = bars, *empty = bars + kInferStages, *acc_full = bars + 6, *act_ready = bars + 7;
    uint64_t *rdx_bar = bars + 8, *drain = bars + 9;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(base + InferSmem::tmem_slot);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(base + InferSmem::abort_flag);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tiles = (P.n + 127) / 128;
    if (warp == 1) tmem_alloc(tmem_slot, 512);
    if (threadIdx.x == 0) {
        for (int s = 0; s < kInferStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(acc_full, 1);
        mbar_init(act_ready, 512);
        mbar_init(rdx_bar, 128);
        mbar_init(drain, 1);
        *abort_flag = 0;
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        // ---------------------------------------------------------------- producer
        if (lane == 0) {
            uint32_t it = 0;
            bool ok = true;
            for (int t = blockIdx.x; ok && t < tiles; t += gridDim.x) {
                for (int m = 0; ok && m < P.members; ++m) {
                    const unsigned char *src = P.packed + static_cast<size_t>(m) * kInferMemberBytes;
                    for (int i = 0; i < kInferTilesPerMember; ++i, ++it) {
                        const uint32_t bytes = i < kInferBigTiles ? 32768u : 16384u;
                        const uint32_t s = it % kInferStages, k = it / kInferStages;
                        if (it >= static_cast<uint32_t>(kInferStages) &&
                            !infer_wait(&empty[s], (k - 1u) & 1u, abort_flag, P.status)) {
                            ok = false;
                            break;
                        }
                        mbar_arrive_expect_tx(&full[s], bytes);
                        bulk_g2s(stages + s * kInferStageBytes, src, bytes, &full[s]);
                        src += bytes;
                    }
                }
            }
            // copies still in flight when a wait gave up: wait (bounded) until they have landed
            if (!ok) {
                const uint32_t first = it > static_cast<uint32_t>(kInferStages) ? it - kInferStages : 0u;
                for (uint32_t j = first; j < it; ++j)
                    mbar_wait(&full[j % kInferStages], (j / kInferStages) & 1u, kInferWaitLimit);
            }
        }
        __syncwarp();
    } else if (warp == 1) {
        // ---------------------------------------------------------------- tensor-core issuer
        if (lane == 0) {
            uint32_t it = 0, layer_no = 0;
            bool ok = true;
            for (int t = blockIdx.x; ok && t < tiles; t += gridDim.x) {
                for (int m = 0; ok && m < P.members; ++m) {
                    for (int l = 0; ok && l < kInferLayers; ++l, ++layer_no) {
                        if (!infer_wait(act_ready, layer_no & 1u, abort_flag, P.status)) {
                            ok = false;
                            break;
                        }
                        tc_fence_after();
                        const int halves = l == 4 ? 1 : 2, kcs = l == 0 ? 1 : 8, nh = l == 4 ? 128 : 256;
                        const uint32_t idesc = umma_idesc_bf16(128, nh);
                        for (int h = 0; ok && h < halves; ++h) {
                            for (int kc = 0; kc < kcs; ++kc, ++it) {
                                const uint32_t s = it % kInferStages, k = it / kInferStages;
                                if (!infer_wait(&full[s], k & 1u, abort_flag, P.status)) {
                                    ok = false;
                                    break;
                                }
                                tc_fence_after();
                                const uint32_t a0 = smem_u32(A + kc * kInferChunkBytes);
                                const uint32_t b0 = smem_u32(stages + s * kInferStageBytes);
#pragma unroll
                                for (int kk = 0; kk < 4; ++kk)
                                    umma_bf16(tmem + static_cast<uint32_t>(h * 256), umma_desc_sw128(a0 + kk * 32),
                                              umma_desc_sw128(b0 + kk * 32), idesc, (kc > 0 || kk > 0) ? 1u : 0u);
                                umma_commit(&empty[s]);
                            }
                        }
                        if (ok) umma_commit(acc_full);
                    }
                }
            }
            if (!ok) {  // let the MMAs already issued finish before the tile memory goes away
                umma_commit(drain);
                mbar_wait(drain, 0u, kInferWaitLimit);
            }
        }
        __syncwarp();
    } else {
        // ---------------------------------------------------------------- epilogue (512 threads)
        const int et = threadIdx.x - 64;
        const int q = warp & 3;            // TMEM lane quarter this warp may read
        const int j = (warp - 2) >> 2;     // column quarter
        const int r = q * 32 + lane;       // query row inside the tile
        const uint32_t lane_addr = tmem + (static_cast<uint32_t>(q * 32) << 16);
        uint32_t layer_no = 0, member_no = 0;
        bool ok = true;
        int t = blockIdx.x;
        if (t < tiles) {
            infer_encode(P, A, t * 128, et);
            epi_release(act_ready);
        }
        for (; ok && t < tiles; t += gridDim.x) {
            float acc[32];
#pragma unroll
            for (int i = 0; i < 32; ++i) acc[i] = 0.0f;
            float s1 = 0.0f, s2 = 0.0f;  // members' R_d on the grid: sum and sum of squares
            for (int m = 0; ok && m < P.members; ++m) {
                const float *bias = P.bias + static_cast<size_t>(m) * kInferBiasPerMember;
                for (int l = 0; l < kInferLayers; ++l, ++layer_no) {
                    // the decision is warp-uniform: tcgen05.ld below is a warp-collective
                    if (!__all_sync(0xffffffffu, infer_wait(acc_full, layer_no & 1u, abort_flag, P.status))) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    if (l < 4) {
                        // hidden layer: columns [128 j, 128 j + 128) of 512, 16 at a time; the bias
                        // as 16-byte vector loads (one address across the warp)
                        const float4 *b4 = reinterpret_cast<const float4 *>(bias + l * kInferHidden);
#pragma unroll 1
                        for (int c0 = j * 128; c0 < j * 128 + 128; c0 += 16) {
                            float4 bb[4];
#pragma unroll
                            for (int i = 0; i < 4; ++i) bb[i] = __ldg(b4 + (c0 >> 2) + i);
                            float v[16];
                            tmem_ld16(lane_addr + static_cast<uint32_t>(c0), v);
                            uint32_t w[8];
#pragma unroll
                            for (int i = 0; i < 4; ++i) {
                                w[2 * i] = pack_bf16x2(infer_gelu(v[4 * i] + bb[i].x), infer_gelu(v[4 * i + 1] + bb[i].y));
                                w[2 * i + 1] =
                                    pack_bf16x2(infer_gelu(v[4 * i + 2] + bb[i].z), infer_gelu(v[4 * i + 3] + bb[i].w));
                            }
                            *reinterpret_cast<uint4 *>(act_unit(A, r, c0)) = make_uint4(w[0], w[1], w[2], w[3]);
                            *reinterpret_cast<uint4 *>(act_unit(A, r, c0 + 8)) = make_uint4(w[4], w[5], w[6], w[7]);
                        }
                        epi_release(act_ready);
                    } else {
                        // output layer: columns [32 j, 32 j + 32) of 128
                        const float *b = bias + 4 * kInferHidden;
                        float rd = 0.0f;
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            float v[16];
                            tmem_ld16(lane_addr + static_cast<uint32_t>(j * 32 + h * 16), v);
#pragma unroll
                            for (int i = 0; i < 16; ++i) {
                                const int c = j * 32 + h * 16 + i;
                                if (c < P.n_out) {
                                    const float y = (v[i] + __ldg(b + c)) * __ldg(P.y_std + c) + __ldg(P.y_mean + c);
                                    acc[h * 16 + i] += y;
                                    if (c < P.nbins) rd += exp10f(y) * __ldg(P.areas + c);
                                }
                            }
                        }
                        // the R_d bins are columns 0..63: quarter 1 hands its partial sums to quarter 0
                        // (two buffers by member parity: a buffer is rewritten two members later,
                        // after quarter 0 has read it and released the member in between)
                        const uint32_t slot = (member_no & 1u) * 128u + static_cast<uint32_t>(r);
                        if (j == 1) {
                            rdx[slot] = rd;
                            mbar_arrive(rdx_bar);
                        } else if (j == 0) {
                            if (!__all_sync(0xffffffffu, infer_wait(rdx_bar, member_no & 1u, abort_flag, P.status))) {
                                ok = false;
                                break;
                            }
                            rd += rdx[slot];
                            s1 += rd;
                            s2 += rd * rd;
                        }
                        ++member_no;
                        const bool last_member = m == P.members - 1;
                        const int next_t = last_member ? t + static_cast<int>(gridDim.x) : t;
                        if (last_member) {
                            const int g = t * 128 + r;
                            if (g < P.n) {
                                const float inv = 1.0f / static_cast<float>(P.members);
                                if (P.out) {
#pragma unroll
                                    for (int i = 0; i < 32; ++i) {
                                        const int c = j * 32 + i;
                                        if (c < P.n_out) P.out[static_cast<size_t>(g) * P.n_out + c] = acc[i] * inv;
                                    }
                                }
                                if (j == 0) {
                                    const float M = static_cast<float>(P.members);
                                    const float mean = s1 / M;
                                    const float var = P.members > 1 ? fmaxf(s2 - s1 * mean, 0.0f) / (M - 1.0f) : 0.0f;
                                    const float sp = sqrtf(var) / fmaxf(mean, 1e-12f);
                                    if (P.rd_mean) P.rd_mean[g] = mean;
                                    if (P.spread) P.spread[g] = sp;
                                    if (P.route) P.route[g] = sp > P.threshold ? 1 : 0;
                                }
                            }
                        }
                        // the activation tile is free (this member's MMAs are done): encode the
                        // next member's (or the next tile's) inputs and hand over
                        if (next_t < tiles) {
                            infer_encode(P, A, next_t * 128, et);
                            epi_release(act_ready);
                        }
                    }
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) tmem_dealloc(tmem, 512);
}

}  // namespace tmc
