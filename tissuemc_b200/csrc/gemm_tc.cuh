// D = A * B^T on the 5th-generation tensor cores (tcgen05), BF16 operands, FP32 accumulation in
// tensor memory, with a fused epilogue. A is M x K and B is N x K, both row-major with K
// contiguous (K-major); K is a multiple of 64. One CTA of 128 threads computes a 128 x BN tile
// over the K range of its blockIdx.z (split-K: each z covers K / gridDim.z, a multiple of 64):
//
//   two shared-memory stages hold 64-wide K slices of A and B in the 128-byte-swizzled K-major
//   layout (umma.cuh). Each thread keeps the next slice's global loads in flight in registers
//   (issued together, before the current slice's MMAs), then stores them into the stage whose
//   MMAs (two slices back) have completed, fences them for the tensor core's async proxy and
//   synchronises; thread 0 issues four tcgen05.mma (K = 16 each) into the TMEM accumulator and
//   commits them to that stage's mbarrier. Every wait is bounded: one that runs out records an
//   error in *status and the results are discarded by the host.
//   The epilogue reads the accumulator with tcgen05.ld (warp w owns TMEM lanes 32w..32w+31, i.e.
//   output rows m0 + 32w + lane), applies the epilogue functor (given the split index) and writes
//   global memory.
#pragma once

#include <cuda_bf16.h>

#include "umma.cuh"

namespace tmc {

constexpr int kGemmBM = 128, kGemmBK = 64, kGemmThreads = 128;
constexpr uint32_t kGemmWaitLimit = 1u << 24;  // mbarrier polls before a wait gives up

template <int BN> struct GemmSmem {
    static constexpr int a_bytes = kGemmBM * 128;  // 128 rows x 64 bf16
    static constexpr int b_bytes = BN * 128;
    static constexpr int stage_bytes = a_bytes + b_bytes;
    static constexpr int bytes = 1024 /*alignment slack*/ + 2 * stage_bytes + 64;
};

// Global loads of one 64-wide K slice of a K-major bf16 matrix: rows [row0, row0 + ROWS), 8
// 16-byte units per row, ROWS * 8 / kGemmThreads units per thread (issued together).
template <int ROWS> struct SliceRegs {
    static constexpr int per_thread = ROWS * 8 / kGemmThreads;
    uint4 v[per_thread];

    __device__ __forceinline__ void load(const __nv_bfloat16 *X, int ld, int nrows_total, int row0, int k0) {
#pragma unroll
        for (int i = 0; i < per_thread; ++i) {
            const int idx = threadIdx.x + i * kGemmThreads;
            const int r = idx >> 3, c = idx & 7;
            v[i] = make_uint4(0u, 0u, 0u, 0u);
            if (row0 + r < nrows_total)
                v[i] = *reinterpret_cast<const uint4 *>(X + static_cast<size_t>(row0 + r) * ld + k0 + c * 8);
        }
    }
    __device__ __forceinline__ void store(unsigned char *tile) const {
#pragma unroll
        for (int i = 0; i < per_thread; ++i) {
            const int idx = threadIdx.x + i * kGemmThreads;
            const int r = idx >> 3, c = idx & 7;
            *reinterpret_cast<uint4 *>(tile + r * 128 + ((c ^ (r & 7)) << 4)) = v[i];
        }
    }
};

// Epilogue functor interface: operator()(split, row, col0, v[8]) for 8 consecutive columns of one
// row (col0 is a multiple of 8; columns at or beyond N must be ignored by the functor).
template <int BN, class Epi>
__global__ void __launch_bounds__(kGemmThreads) gemm_tc_kernel(const __nv_bfloat16 *__restrict__ A,
                                                              const __nv_bfloat16 *__restrict__ B, int M, int N,
                                                              int K, Epi epi, int *status) {
    extern __shared__ unsigned char gsm_raw[];
    unsigned char *base = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(gsm_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    uint64_t *bar = reinterpret_cast<uint64_t *>(base + 2 * GemmSmem<BN>::stage_bytes);  // [2]
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bar + 2);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.y * kGemmBM, n0 = blockIdx.x * BN;
    if (warp == 0) tmem_alloc(tmem_slot, BN);
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_d = *tmem_slot;
    constexpr uint32_t idesc = umma_idesc_bf16(kGemmBM, BN);

    const int kt_n = K / kGemmBK / static_cast<int>(gridDim.z);  // K slices of this split
    const int kt0 = static_cast<int>(blockIdx.z) * kt_n;
    SliceRegs<kGemmBM> ra;
    SliceRegs<BN> rb;
    ra.load(A, K, M, m0, kt0 * kGemmBK);
    rb.load(B, K, N, n0, kt0 * kGemmBK);
    bool ok = true;
    for (int kt = 0; kt < kt_n; ++kt) {
        const int s = kt & 1;
        unsigned char *sa = base + s * GemmSmem<BN>::stage_bytes;
        unsigned char *sb = sa + GemmSmem<BN>::a_bytes;
        // the stage was last read by the MMAs of slice kt - 2
        if (kt >= 2 && ok && !mbar_wait(&bar[s], static_cast<uint32_t>(((kt - 2) >> 1) & 1), kGemmWaitLimit)) {
            ok = false;
            atomicExch(status, 1);
        }
        ra.store(sa);
        rb.store(sb);
        fence_async_smem();
        __syncthreads();
        if (kt + 1 < kt_n) {  // the next slice's loads fly while this slice's MMAs run
            ra.load(A, K, M, m0, (kt0 + kt + 1) * kGemmBK);
            rb.load(B, K, N, n0, (kt0 + kt + 1) * kGemmBK);
        }
        if (threadIdx.x == 0) {
            tc_fence_after();
            const uint32_t a0 = smem_u32(sa), b0 = smem_u32(sb);
#pragma unroll
            for (int kk = 0; kk < kGemmBK / 16; ++kk)  // 16 bf16 = 32 bytes further along K
                umma_bf16(tmem_d, umma_desc_sw128(a0 + kk * 32), umma_desc_sw128(b0 + kk * 32), idesc,
                          (kt > 0 || kk > 0) ? 1u : 0u);
            umma_commit(&bar[s]);
        }
    }
    // the last commit completes when every MMA of the tile has
    const int last = kt_n - 1;
    if (ok && !mbar_wait(&bar[last & 1], static_cast<uint32_t>((last >> 1) & 1), kGemmWaitLimit)) {
        ok = false;
        atomicExch(status, 1);
    }
    tc_fence_after();
    ok = __all_sync(0xffffffffu, ok);  // tcgen05.ld is warp-collective
    if (ok) {
        const int row = m0 + warp * 32 + lane;
        const uint32_t lane_addr = tmem_d + (static_cast<uint32_t>(warp * 32) << 16);
#pragma unroll 1
        for (int c = 0; c < BN; c += 8) {
            float v[8];
            tmem_ld8(lane_addr + static_cast<uint32_t>(c), v);
            if (row < M && n0 + c < N) epi(static_cast<int>(blockIdx.z), row, n0 + c, v);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem_d, BN);
}

}  // namespace tmc
