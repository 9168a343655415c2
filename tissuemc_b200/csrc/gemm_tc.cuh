// D = A * B^T on the 5th-generation tensor cores (tcgen05), BF16 operands, FP32 accumulation in
// tensor memory, with a fused epilogue. A is M x K and B is N x K, both row-major with K
// contiguous (K-major), 16-byte aligned; K is a multiple of 64. One CTA of four warps computes a
// 128 x BN tile over the K range of its blockIdx.z (split-K: each z covers K / gridDim.z, a
// multiple of 64):
//
//   warp 0 (the producer) streams 64-wide K slices of A and B into a ring of kGemmStages
//   shared-memory stages with tiled TMA loads (cp.async.bulk.tensor, 128-byte swizzle: the layout
//   the MMA descriptors read, umma.cuh), each stage's mbarrier counting the bytes in; warp 1 (the
//   issuer) waits for a stage, issues its four tcgen05.mma (K = 16 each) into the TMEM accumulator
//   and commits them to the stage's "empty" mbarrier, which hands the stage back to the producer;
//   a last commit marks the accumulator complete. Rows past M or N arrive as zeros. Every wait is
//   bounded: one that runs out records an error in *status (the host discards the results) and
//   the CTA skips its epilogue. Nothing is released while this CTA's own asynchronous work may
//   still be in flight: the issuer commits the accumulator barrier after whatever MMAs it issued
//   (also when it gave up), every warp waits for that barrier before TMEM is read or freed, and
//   the producer waits for every load it issued; these drain waits have a longer limit of their
//   own (issued copies and MMAs finish without help from any other party). Only if a drain wait
//   runs out too does the CTA free TMEM regardless (so that a later CTA can allocate it) and
//   report status 2.
//   The epilogue reads the accumulator with tcgen05.ld, 32 columns per load (warp w owns TMEM
//   lanes 32w..32w+31, i.e. output rows m0 + 32w + lane), applies the epilogue functor (given the
//   split index) to each 8 columns and writes global memory.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>

#include "umma.cuh"

namespace tmc {

constexpr int kGemmBM = 128, kGemmBK = 64, kGemmThreads = 128, kGemmStages = 3;
constexpr uint32_t kGemmWaitLimit = 1u << 24;   // mbarrier polls before a wait gives up
constexpr uint32_t kGemmDrainLimit = 1u << 26;  // polls of a wait for this CTA's own issued work

template <int BN> struct GemmSmem {
    static constexpr int a_bytes = kGemmBM * 128;  // 128 rows x 64 bf16
    static constexpr int b_bytes = BN * 128;
    static constexpr int stage_bytes = a_bytes + b_bytes;
    // alignment slack, the stages, then 2 x kGemmStages + 1 mbarriers, the TMEM address and the
    // CTA's abort flag
    static constexpr int bytes = 1024 + kGemmStages * stage_bytes + 128;
};

// Epilogue functor interface: operator()(split, row, col0, v[8]) for 8 consecutive columns of one
// row (col0 is a multiple of 8; columns at or beyond N must be ignored by the functor).
// wait_limit bounds the waits on the other roles (kGemmWaitLimit in production). withhold = 1 is
// a test of the give-up path: the producer issues no loads, so the issuer's first wait runs out
// with no copy and no MMA outstanding.
template <int BN, class Epi>
__global__ void __launch_bounds__(kGemmThreads) gemm_tc_kernel(const __grid_constant__ CUtensorMap tma_a,
                                                              const __grid_constant__ CUtensorMap tma_b, int M, int N,
                                                              int K, Epi epi, int *status, uint32_t wait_limit,
                                                              int withhold) {
    static_assert(GemmSmem<BN>::a_bytes % 1024 == 0 && GemmSmem<BN>::b_bytes % 1024 == 0, "1024-byte tiles");
    extern __shared__ unsigned char gsm_raw[];
    unsigned char *base = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(gsm_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    uint64_t *full = reinterpret_cast<uint64_t *>(base + kGemmStages * GemmSmem<BN>::stage_bytes);
    uint64_t *empty = full + kGemmStages;
    uint64_t *acc_bar = empty + kGemmStages;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(acc_bar + 1);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.y * kGemmBM, n0 = blockIdx.x * BN;
    if (warp == 0) tmem_alloc(tmem_slot, BN);
    if (threadIdx.x == 0) {
        for (int s = 0; s < kGemmStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(acc_bar, 1);
        *abort_flag = 0;
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_d = *tmem_slot;
    constexpr uint32_t idesc = umma_idesc_bf16(kGemmBM, BN);

    const int kt_n = K / kGemmBK / static_cast<int>(gridDim.z);  // K slices of this split
    const int kt0 = static_cast<int>(blockIdx.z) * kt_n;
    bool ok = true;
    if (warp == 0) {
        // ---- producer: the whole warp walks the ring, lane 0 issues
        int issued = 0;
        for (int kt = 0; kt < (withhold ? 0 : kt_n); ++kt) {
            const int s = kt % kGemmStages;
            // the stage was last read by the MMAs of slice kt - kGemmStages
            if (kt >= kGemmStages &&
                !mbar_wait(&empty[s], static_cast<uint32_t>((kt / kGemmStages - 1) & 1), wait_limit)) {
                ok = false;
                break;
            }
            if (lane == 0) {
                unsigned char *sa = base + s * GemmSmem<BN>::stage_bytes;
                mbar_arrive_expect_tx(&full[s], GemmSmem<BN>::stage_bytes);
                tma_load_2d(sa, &tma_a, (kt0 + kt) * kGemmBK, m0, &full[s]);
                tma_load_2d(sa + GemmSmem<BN>::a_bytes, &tma_b, (kt0 + kt) * kGemmBK, n0, &full[s]);
            }
            __syncwarp();
            issued = kt + 1;
        }
        // every load issued has landed before the CTA can end (the last phase of each stage)
        for (int kt = issued > kGemmStages ? issued - kGemmStages : 0; kt < issued; ++kt)
            if (!mbar_wait(&full[kt % kGemmStages], static_cast<uint32_t>((kt / kGemmStages) & 1), kGemmDrainLimit)) {
                ok = false;
                if (lane == 0) atomicExch(status, 2);
            }
    } else if (warp == 1) {
        // ---- issuer: the whole warp waits, lane 0 issues the MMAs and the commits
        for (int kt = 0; kt < kt_n; ++kt) {
            const int s = kt % kGemmStages;
            if (!mbar_wait(&full[s], static_cast<uint32_t>((kt / kGemmStages) & 1), wait_limit)) {
                ok = false;
                break;
            }
            tc_fence_after();
            if (lane == 0) {
                const uint32_t a0 = smem_u32(base + s * GemmSmem<BN>::stage_bytes);
                const uint32_t b0 = a0 + GemmSmem<BN>::a_bytes;
#pragma unroll
                for (int kk = 0; kk < kGemmBK / 16; ++kk)  // 16 bf16 = 32 bytes further along K
                    umma_bf16(tmem_d, umma_desc_sw128(a0 + kk * 32), umma_desc_sw128(b0 + kk * 32), idesc,
                              (kt > 0 || kk > 0) ? 1u : 0u);
                umma_commit(&empty[s]);
            }
            __syncwarp();
        }
        // arrives when every MMA issued above has completed, also after a give-up
        if (lane == 0) umma_commit(acc_bar);
        __syncwarp();
    }
    if (!ok) {
        if (lane == 0) atomicCAS(status, 0, 1);
        *abort_flag = 1;
    }
    // every MMA this CTA issued has completed before TMEM is read or released
    if (!mbar_wait(acc_bar, 0u, wait_limit)) {
        if (lane == 0) atomicCAS(status, 0, 1);
        *abort_flag = 1;
        if (!mbar_wait(acc_bar, 0u, kGemmDrainLimit) && lane == 0) atomicExch(status, 2);
    }
    tc_fence_after();
    __syncthreads();                 // orders the abort flag: the epilogue runs in every warp or none
    ok = *abort_flag == 0;
    if (ok) {
        const int row = m0 + warp * 32 + lane;
        const uint32_t lane_addr = tmem_d + (static_cast<uint32_t>(warp * 32) << 16);
        static_assert(BN % 32 == 0, "the epilogue reads 32 accumulator columns at a time");
#pragma unroll 1
        for (int c = 0; c < BN; c += 32) {
            float v[32];
            tmem_ld32(lane_addr + static_cast<uint32_t>(c), v);
            if (row < M) {
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    if (n0 + c + 8 * q < N)
                        epi(static_cast<int>(blockIdx.z), row, n0 + c + 8 * q,
                            *reinterpret_cast<const float(*)[8]>(v + 8 * q));
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem_d, BN);
}

}  // namespace tmc
