// D = A * B^T on the 5th-generation tensor cores (tcgen05), BF16 operands, FP32 accumulation in
// tensor memory, with a fused epilogue. A is M x K and B is N x K, both row-major with K
// contiguous (K-major); K is a multiple of 64. One CTA of 128 threads computes a 128 x BN tile:
//
//   for each 64-wide K slice: all threads stage the A and B slices in shared memory in the
//   128-byte-swizzled K-major layout (umma.cuh), fence them for the tensor core's async proxy and
//   synchronise; thread 0 issues four tcgen05.mma (K = 16 each) into the TMEM accumulator and
//   commits them to an mbarrier; every thread waits on the mbarrier (bounded: a wait that runs
//   out records an error in *status and the results are discarded by the host) before the next
//   slice overwrites shared memory.
//   The epilogue reads the accumulator with tcgen05.ld (warp w owns TMEM lanes 32w..32w+31, i.e.
//   output rows m0 + 32w + lane), applies the epilogue functor and writes global memory.
#pragma once

#include <cuda_bf16.h>

#include "umma.cuh"

namespace tmc {

constexpr int kGemmBM = 128, kGemmBK = 64, kGemmThreads = 128;
constexpr uint32_t kGemmWaitLimit = 1u << 24;  // mbarrier polls before a wait gives up

template <int BN> struct GemmSmem {
    static constexpr int a_bytes = kGemmBM * 128;  // 128 rows x 64 bf16
    static constexpr int b_bytes = BN * 128;
    static constexpr int bytes = 1024 /*alignment slack*/ + a_bytes + b_bytes + 64;
};

// Stage rows [row0, row0 + rows) x K slice [k0, k0 + 64) of a K-major bf16 matrix into a swizzled tile.
__device__ __forceinline__ void stage_tile(unsigned char *tile, const __nv_bfloat16 *X, int ld, int nrows_total,
                                          int row0, int rows, int k0) {
    for (int idx = threadIdx.x; idx < rows * 8; idx += kGemmThreads) {
        const int r = idx >> 3, c = idx & 7;
        uint4 v = make_uint4(0u, 0u, 0u, 0u);
        if (row0 + r < nrows_total)
            v = *reinterpret_cast<const uint4 *>(X + static_cast<size_t>(row0 + r) * ld + k0 + c * 8);
        *reinterpret_cast<uint4 *>(tile + r * 128 + ((c ^ (r & 7)) << 4)) = v;
    }
}

// Epilogue functor interface: operator()(row, col0, v[8]) for 8 consecutive columns of one row
// (col0 is a multiple of 8; columns at or beyond N must be ignored by the functor).
template <int BN, class Epi>
__global__ void __launch_bounds__(kGemmThreads) gemm_tc_kernel(const __nv_bfloat16 *__restrict__ A,
                                                              const __nv_bfloat16 *__restrict__ B, int M, int N,
                                                              int K, Epi epi, int *status) {
    extern __shared__ unsigned char gsm_raw[];
    unsigned char *base = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(gsm_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    unsigned char *sa = base;
    unsigned char *sb = base + GemmSmem<BN>::a_bytes;
    uint64_t *bar = reinterpret_cast<uint64_t *>(sb + GemmSmem<BN>::b_bytes);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bar + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.y * kGemmBM, n0 = blockIdx.x * BN;
    if (warp == 0) tmem_alloc(tmem_slot, BN);
    if (threadIdx.x == 0) mbar_init(bar, 1);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_d = *tmem_slot;
    constexpr uint32_t idesc = umma_idesc_bf16(kGemmBM, BN);

    bool ok = true;
    const int kt_n = K / kGemmBK;
    for (int kt = 0; kt < kt_n; ++kt) {
        stage_tile(sa, A, K, M, m0, kGemmBM, kt * kGemmBK);
        stage_tile(sb, B, K, N, n0, BN, kt * kGemmBK);
        fence_async_smem();
        __syncthreads();
        if (threadIdx.x == 0) {
            tc_fence_after();
            const uint32_t a0 = smem_u32(sa), b0 = smem_u32(sb);
#pragma unroll
            for (int kk = 0; kk < kGemmBK / 16; ++kk)  // 16 bf16 = 32 bytes further along K
                umma_bf16(tmem_d, umma_desc_sw128(a0 + kk * 32), umma_desc_sw128(b0 + kk * 32), idesc,
                          (kt > 0 || kk > 0) ? 1u : 0u);
            umma_commit(bar);
        }
        if (ok && !mbar_wait(bar, static_cast<uint32_t>(kt & 1), kGemmWaitLimit)) {
            ok = false;
            atomicExch(status, 1);
        }
        __syncthreads();
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
            if (row < M && n0 + c < N) epi(row, n0 + c, v);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem_d, BN);
}

}  // namespace tmc
