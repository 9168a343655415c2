// The surrogate's neural-network kernels and their C ABI (no counterpart in the reference: the
// learned surrogate is an addition of this engine). Every matrix product runs on the tcgen05
// tensor cores through gemm_tc.cuh (BF16 operands, FP32 accumulation in tensor memory) with the
// bias, GELU and GELU-derivative work fused into its epilogue; the element-wise kernels (transpose,
// bias gradient, loss, Adam) are plain CUDA. Entry points take device pointers and a stream and
// do not synchronise (so a training step can be captured in a CUDA graph); a bounded tensor-core
// wait that gives up sets a per-device status word read by tmc_b200_nn_status.

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/tissuemc_b200.h"
#include "gemm_tc.cuh"
#include "mlp_infer.cuh"

namespace tmc {
namespace {

constexpr int kBN = 128;
// three stages of 32 KB plus slack: two CTAs per SM, i.e. 2 x 128 of the 512 TMEM columns
constexpr int kGemmSmemRequest = GemmSmem<kBN>::bytes;
static_assert(2 * kGemmSmemRequest <= 227 * 1024, "two GEMM CTAs per SM");

__device__ __forceinline__ float gelu(float x) { return gelu_tanh(x); }
__device__ __forceinline__ float gelu_grad(float x) { return gelu_tanh_grad(x); }

// Eight consecutive columns of a row start on a 16-byte boundary when the row length is a multiple
// of 8 (bf16) / 4 (float32); then the epilogues move them with vector loads and stores (one
// instruction per 8 bf16 or 4 floats instead of one per element).
__device__ __forceinline__ uint4 pack8_bf16(const float (&x)[8]) {
    uint4 u;
    __nv_bfloat162 h;
    h = __floats2bfloat162_rn(x[0], x[1]);
    u.x = *reinterpret_cast<const uint32_t *>(&h);
    h = __floats2bfloat162_rn(x[2], x[3]);
    u.y = *reinterpret_cast<const uint32_t *>(&h);
    h = __floats2bfloat162_rn(x[4], x[5]);
    u.z = *reinterpret_cast<const uint32_t *>(&h);
    h = __floats2bfloat162_rn(x[6], x[7]);
    u.w = *reinterpret_cast<const uint32_t *>(&h);
    return u;
}

// D (float32) = acc (+ bias); split z of a split-K product writes its partial at D + z * split_stride
struct EpiF32 {
    float *D;
    const float *bias;
    int N;
    size_t split_stride;
    __device__ __forceinline__ void operator()(int split, int row, int col, const float (&v)[8]) const {
        float *d = D + split * split_stride + static_cast<size_t>(row) * N + col;
        float x[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) x[i] = v[i] + ((bias && col + i < N) ? bias[col + i] : 0.0f);
        if (N % 4 == 0 && col + 8 <= N) {
            reinterpret_cast<float4 *>(d)[0] = make_float4(x[0], x[1], x[2], x[3]);
            reinterpret_cast<float4 *>(d)[1] = make_float4(x[4], x[5], x[6], x[7]);
        } else {
#pragma unroll
            for (int i = 0; i < 8; ++i)
                if (col + i < N) d[i] = x[i];
        }
    }
};

// h (bf16) also into HT, the transpose (N x M): lane = row, so a warp's stores of one column are
// 32 consecutive bf16 (coalesced); this replaces a separate transpose pass.
__device__ __forceinline__ void store_transposed(__nv_bfloat16 *HT, int M, int N, int row, int col,
                                                 const float (&h)[8]) {
#pragma unroll
    for (int i = 0; i < 8; ++i)
        if (col + i < N) HT[static_cast<size_t>(col + i) * M + row] = __float2bfloat16_rn(h[i]);
}

// Forward linear layer: z = acc + bias (stored as float32 if Z), h = act(z) (stored as bf16 if H,
// and transposed as bf16 if HT, an N x M matrix).
struct EpiFwd {
    const float *bias;
    float *Z;
    __nv_bfloat16 *H;
    int N, act;
    __nv_bfloat16 *HT;
    int M;
    __device__ __forceinline__ void operator()(int, int row, int col, const float (&v)[8]) const {
        const size_t o = static_cast<size_t>(row) * N + col;
        float z[8], h[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            z[i] = v[i] + (col + i < N ? bias[col + i] : 0.0f);
            h[i] = act ? gelu(z[i]) : z[i];
        }
        if (HT) store_transposed(HT, M, N, row, col, h);
        if (N % 8 == 0 && col + 8 <= N) {
            if (Z) {
                reinterpret_cast<float4 *>(Z + o)[0] = make_float4(z[0], z[1], z[2], z[3]);
                reinterpret_cast<float4 *>(Z + o)[1] = make_float4(z[4], z[5], z[6], z[7]);
            }
            if (H) *reinterpret_cast<uint4 *>(H + o) = pack8_bf16(h);
        } else {
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                if (col + i >= N) break;
                if (Z) Z[o + i] = z[i];
                if (H) H[o + i] = __float2bfloat16_rn(h[i]);
            }
        }
    }
};

// Backward through a linear layer into the previous GELU: dx = acc * gelu'(z_prev), bf16 (and
// transposed into dXT, an N x M matrix, if given).
struct EpiBwd {
    const float *Zprev;
    __nv_bfloat16 *dX;
    int N;
    __nv_bfloat16 *dXT;
    int M;
    __device__ __forceinline__ void operator()(int, int row, int col, const float (&v)[8]) const {
        const size_t o = static_cast<size_t>(row) * N + col;
        float d[8];
        if (N % 8 == 0 && col + 8 <= N) {
            const float4 z0 = reinterpret_cast<const float4 *>(Zprev + o)[0];
            const float4 z1 = reinterpret_cast<const float4 *>(Zprev + o)[1];
            const float z[8] = {z0.x, z0.y, z0.z, z0.w, z1.x, z1.y, z1.z, z1.w};
#pragma unroll
            for (int i = 0; i < 8; ++i) d[i] = v[i] * gelu_grad(z[i]);
            *reinterpret_cast<uint4 *>(dX + o) = pack8_bf16(d);
        } else {
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                d[i] = col + i < N ? v[i] * gelu_grad(Zprev[o + i]) : 0.0f;
                if (col + i < N) dX[o + i] = __float2bfloat16_rn(d[i]);
            }
        }
        if (dXT) store_transposed(dXT, M, N, row, col, d);
    }
};

__global__ void transpose_bf16_kernel(const __nv_bfloat16 *__restrict__ X, __nv_bfloat16 *__restrict__ Y, int rows,
                                      int cols) {
    __shared__ __nv_bfloat16 tile[32][33];
    const int c = blockIdx.x * 32 + threadIdx.x, r0 = blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += blockDim.y)
        if (r0 + j < rows && c < cols) tile[j][threadIdx.x] = X[static_cast<size_t>(r0 + j) * cols + c];
    __syncthreads();
    const int r = blockIdx.y * 32 + threadIdx.x, c0 = blockIdx.x * 32;
    for (int j = threadIdx.y; j < 32; j += blockDim.y)
        if (c0 + j < cols && r < rows) Y[static_cast<size_t>(c0 + j) * rows + r] = tile[threadIdx.x][j];
}

// Bias gradient db[n] = sum over rows of dZ[row][n], deterministically in two passes: block row y
// of the first sums rows y, y + G, y + 2G, ... (G = kColsumGroups) of its 128 columns into
// part[y][n]; the second adds the G partial sums of each column in a fixed order. No atomics, so a
// training step gives the same bits every time it runs.
constexpr int kColsumGroups = 128;

__global__ void colsum_partial_kernel(const __nv_bfloat16 *__restrict__ dZ, float *__restrict__ part, int M, int N) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    float s[4] = {0.0f, 0.0f, 0.0f, 0.0f};  // four independent chains keep several loads in flight
    int m = blockIdx.y;
    for (; m + 3 * static_cast<int>(gridDim.y) < M; m += 4 * gridDim.y) {
#pragma unroll
        for (int u = 0; u < 4; ++u) s[u] += __bfloat162float(dZ[static_cast<size_t>(m + u * gridDim.y) * N + n]);
    }
    for (; m < M; m += gridDim.y) s[0] += __bfloat162float(dZ[static_cast<size_t>(m) * N + n]);
    part[static_cast<size_t>(blockIdx.y) * N + n] = (s[0] + s[1]) + (s[2] + s[3]);
}

// One warp per column: lane l adds partial rows l, l + 32, ... in order, then a fixed shuffle tree
// adds the lanes (deterministic, and 32 loads in flight per column instead of one).
__global__ void colsum_final_kernel(const float *__restrict__ part, float *__restrict__ db, int N, int groups) {
    const int n = static_cast<int>((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (n >= N) return;  // warp-uniform
    float acc = 0.0f;
    for (int y = lane; y < groups; y += 32) acc += part[static_cast<size_t>(y) * N + n];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) db[n] = acc;
}

// Mean-squared error over the first T of ld columns: loss += scale * sum (p - t)^2 and
// dZ = 2 * scale * (p - t) (bf16; zero in the padded columns). Grid-stride over the elements; each
// block adds its partial loss once (one atomic per block rather than per warp).
__global__ void mse_kernel(const float *__restrict__ pred, const float *__restrict__ target, __nv_bfloat16 *dZ,
                           float *loss, int M, int T, int ld, float scale) {
    __shared__ float warp_sum[32];
    const size_t n = static_cast<size_t>(M) * ld;
    float l = 0.0f;
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int row = static_cast<int>(i / ld), col = static_cast<int>(i % ld);
        float g = 0.0f;
        if (col < T) {
            const float d = pred[i] - target[static_cast<size_t>(row) * T + col];
            l += d * d;
            g = 2.0f * scale * d;
        }
        if (dZ) dZ[i] = __float2bfloat16_rn(g);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) warp_sum[threadIdx.x >> 5] = l;
    __syncthreads();
    if (threadIdx.x < 32) {
        l = threadIdx.x < (blockDim.x >> 5) ? warp_sum[threadIdx.x] : 0.0f;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
        if (threadIdx.x == 0 && l != 0.0f) atomicAdd(loss, l * scale);
    }
}

// Polyak averaging of one value: avg = beta avg + (1 - beta) w, with its rounding pinned so that
// the separate pass (ema_kernel) and the one fused into Adam give the same bits.
__device__ __forceinline__ float polyak(float avg, float w, float beta) {
    return __fmaf_rn(beta, avg, __fmul_rn(__fsub_rn(1.0f, beta), w));
}

// One Adam step of element i of a rows x cols float32 parameter (row-major): the moments, the
// weight, its Polyak average (if avg), its bf16 copy (if wb) and transpose (if wt). Shared by the
// one-tensor and the many-tensor kernels, so both give the same bits.
__device__ __forceinline__ void adam_element(size_t i, float *__restrict__ w, const float *__restrict__ g,
                                             float *__restrict__ m, float *__restrict__ v, int rows, int cols,
                                             float lr, float b1, float b2, float eps, float weight_decay,
                                             __nv_bfloat16 *wb, __nv_bfloat16 *wt, float *__restrict__ avg,
                                             float avg_beta) {
    const float gi = g[i] + weight_decay * w[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * mi / (sqrtf(vi) + eps);
    w[i] = wi;
    if (avg) avg[i] = polyak(avg[i], wi, avg_beta);
    const __nv_bfloat16 b = __float2bfloat16_rn(wi);
    if (wb) wb[i] = b;
    if (wt) {
        const int r = static_cast<int>(i / cols), c = static_cast<int>(i % cols);
        wt[static_cast<size_t>(c) * rows + r] = b;
    }
}

// Adam on float32 master weights (rows x cols, row-major), writing the bf16 copy and its transpose.
// The step size is lr_dev[0] when lr_dev is given (so that a captured graph reads the current
// step's value), else lr_t; with avg given, the averaged weights are updated from the new ones.
__global__ void adam_kernel(float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m,
                            float *__restrict__ v, int rows, int cols, float lr_t, const float *__restrict__ lr_dev,
                            float b1, float b2, float eps, float weight_decay, __nv_bfloat16 *wb,
                            __nv_bfloat16 *wt, float *__restrict__ avg, float avg_beta) {
    const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= static_cast<size_t>(rows) * cols) return;
    const float lr = lr_dev ? __ldg(lr_dev) : lr_t;
    adam_element(i, w, g, m, v, rows, cols, lr, b1, b2, eps, weight_decay, wb, wt, avg, avg_beta);
}

constexpr int kAdamThreads = 256;

// The same step for every tensor of a table (one launch for all of a network's parameters): block b
// belongs to the tensor whose first_block range holds it.
__global__ void adam_multi_kernel(const tmc_adam_tensor *__restrict__ tab, int count, float lr_t,
                                  const float *__restrict__ lr_dev, float b1, float b2, float eps, float avg_beta) {
    __shared__ tmc_adam_tensor T;
    if (threadIdx.x == 0) {
        int t = 0;
        while (t + 1 < count && static_cast<int>(blockIdx.x) >= tab[t + 1].first_block) ++t;
        T = tab[t];
    }
    __syncthreads();
    const size_t i = static_cast<size_t>(static_cast<int>(blockIdx.x) - T.first_block) * kAdamThreads + threadIdx.x;
    if (i >= static_cast<size_t>(T.rows) * T.cols) return;
    const float lr = lr_dev ? __ldg(lr_dev) : lr_t;
    adam_element(i, T.w, T.g, T.m, T.v, T.rows, T.cols, lr, b1, b2, eps, T.weight_decay,
                 reinterpret_cast<__nv_bfloat16 *>(T.wb), reinterpret_cast<__nv_bfloat16 *>(T.wt), T.avg, avg_beta);
}

// D = sum over the splits of a split-K product's partials (fixed order: deterministic)
__global__ void sum_splits_kernel(const float *__restrict__ work, float *__restrict__ D, size_t n, int splits) {
    const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float acc = 0.0f;
    for (int z = 0; z < splits; ++z) acc += work[z * n + i];
    D[i] = acc;
}

__global__ void ema_kernel(const float *__restrict__ w, float *__restrict__ avg, size_t n, float beta) {
    const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) avg[i] = polyak(avg[i], w[i], beta);
}

__global__ void to_bf16_kernel(const float *__restrict__ w, int rows, int cols, __nv_bfloat16 *wb,
                               __nv_bfloat16 *wt) {
    const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= static_cast<size_t>(rows) * cols) return;
    const __nv_bfloat16 b = __float2bfloat16_rn(w[i]);
    if (wb) wb[i] = b;
    if (wt) wt[static_cast<size_t>(i % cols) * rows + i / cols] = b;
}

// Network inputs from raw features: z-score the first nf of n_feat columns, zero-pad to ld, bf16.
__global__ void encode_kernel(const float *__restrict__ feats, const float *__restrict__ mean,
                              const float *__restrict__ stdv, __nv_bfloat16 *__restrict__ X, int n, int nf, int ld) {
    const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= static_cast<size_t>(n) * ld) return;
    const int row = static_cast<int>(i / ld), col = static_cast<int>(i % ld);
    const float v = col < nf ? (feats[static_cast<size_t>(row) * nf + col] - mean[col]) / stdv[col] : 0.0f;
    X[i] = __float2bfloat16_rn(v);
}

// The ensemble gate: for each query, every member's diffuse reflectance on the grid
// (sum over bins of 10^(z * std + mean) * area), their mean, their spread (sample standard
// deviation over the mean) and whether the spread exceeds the threshold (route the query to Monte
// Carlo).
__global__ void gate_kernel(const float *__restrict__ Z, int members, size_t member_stride, int ld,
                            const float *__restrict__ ymean, const float *__restrict__ ystd,
                            const float *__restrict__ areas, int nbins, int n, float threshold, float *rd_mean,
                            float *spread, unsigned char *route) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    float s1 = 0.0f, s2 = 0.0f;
    for (int m = 0; m < members; ++m) {
        const float *z = Z + m * member_stride + static_cast<size_t>(q) * ld;
        float rd = 0.0f;
        for (int b = 0; b < nbins; ++b) rd += exp10f(z[b] * ystd[b] + ymean[b]) * areas[b];
        s1 += rd;
        s2 += rd * rd;
    }
    const float mean = s1 / members;
    const float var = members > 1 ? fmaxf(s2 - s1 * mean, 0.0f) / (members - 1) : 0.0f;
    const float sp = sqrtf(var) / fmaxf(mean, 1e-12f);
    if (rd_mean) rd_mean[q] = mean;
    if (spread) spread[q] = sp;
    route[q] = sp > threshold ? 1 : 0;
}

std::mutex g_mu;
int *g_status[64] = {};
bool g_attr[64] = {};
bool g_infer_attr[64] = {};

void put(tmc_status *st, int code, const std::string &m) {
    if (!st) return;
    st->code = code;
    std::snprintf(st->message, sizeof st->message, "%s", m.c_str());
}

int current_device() {
    int d = -1;
    if (cudaGetDevice(&d) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    return d;
}

// The per-device status word (allocated at the first call on a device, before any capture).
int *status_word(int dev) {
    if (dev < 0 || dev >= 64) return nullptr;
    if (!g_status[dev]) {
        if (cudaMalloc(&g_status[dev], sizeof(int)) != cudaSuccess) return nullptr;
        if (cudaMemset(g_status[dev], 0, sizeof(int)) != cudaSuccess) return nullptr;
    }
    return g_status[dev];
}

template <class Epi> void set_smem_attr() {
    cudaFuncSetAttribute(gemm_tc_kernel<kBN, Epi>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGemmSmemRequest);
}

// cuTensorMapEncodeTiled, from the driver through the runtime (no link against libcuda).
PFN_cuTensorMapEncodeTiled_v12000 g_encode_tiled = nullptr;

// Tensor map of a rows x K bf16 matrix (K contiguous) read in boxes of 64 (K) x box_rows, with the
// 128-byte swizzle of the MMA operand tiles; rows past the end read as zeros.
bool encode_operand(CUtensorMap *map, const void *ptr, int rows, int K, int box_rows) {
    const cuuint64_t dims[2] = {static_cast<cuuint64_t>(K), static_cast<cuuint64_t>(rows)};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(K) * 2u};
    const cuuint32_t box[2] = {static_cast<cuuint32_t>(kGemmBK), static_cast<cuuint32_t>(box_rows)};
    const cuuint32_t elem[2] = {1u, 1u};
    return g_encode_tiled(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(ptr), dims, strides, box, elem,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Common checks and the launch of one tensor-core GEMM (asynchronous).
template <class Epi>
int launch_gemm(const void *A, const void *B, int M, int N, int K, const Epi &epi, void *stream, tmc_status *st,
                int splits = 1, uint32_t wait_limit = kGemmWaitLimit, int withhold = 0) {
    if (!A || !B) {
        put(st, TMC_BAD_ARGUMENT, "NULL argument");
        return TMC_BAD_ARGUMENT;
    }
    if (M < 1 || N < 1 || K < 64 || K % 64 != 0) {
        put(st, TMC_BAD_CONFIG, "tensor-core GEMM needs M, N >= 1 and K a positive multiple of 64");
        return TMC_BAD_CONFIG;
    }
    if (splits < 1 || (K / 64) % splits != 0) {
        put(st, TMC_BAD_CONFIG, "split-K needs K / 64 to be a multiple of the number of splits");
        return TMC_BAD_CONFIG;
    }
    if (reinterpret_cast<uintptr_t>(A) % 16 != 0 || reinterpret_cast<uintptr_t>(B) % 16 != 0) {
        put(st, TMC_BAD_ARGUMENT, "tensor-core GEMM operands must be 16-byte aligned");
        return TMC_BAD_ARGUMENT;
    }
    const int dev = current_device();
    std::lock_guard<std::mutex> lock(g_mu);
    int *status = status_word(dev);
    if (!status) {
        put(st, TMC_NO_DEVICE, "no usable CUDA device found");
        return TMC_NO_DEVICE;
    }
    if (!g_encode_tiled) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn) {
            cudaGetLastError();
            put(st, TMC_CUDA_ERROR, "the CUDA driver does not provide cuTensorMapEncodeTiled");
            return TMC_CUDA_ERROR;
        }
        g_encode_tiled = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    if (!g_attr[dev]) {
        set_smem_attr<EpiF32>();
        set_smem_attr<EpiFwd>();
        set_smem_attr<EpiBwd>();
        g_attr[dev] = true;
    }
    CUtensorMap ta, tb;
    if (!encode_operand(&ta, A, M, K, kGemmBM) || !encode_operand(&tb, B, N, K, kBN)) {
        put(st, TMC_BAD_ARGUMENT, "tensor-core GEMM operands do not fit a TMA tensor map");
        return TMC_BAD_ARGUMENT;
    }
    const dim3 grid((N + kBN - 1) / kBN, (M + kGemmBM - 1) / kGemmBM, splits);
    gemm_tc_kernel<kBN, Epi><<<grid, kGemmThreads, kGemmSmemRequest, static_cast<cudaStream_t>(stream)>>>(
        ta, tb, M, N, K, epi, status, wait_limit, withhold);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        put(st, TMC_CUDA_ERROR, std::string("CUDA error launching the tensor-core GEMM: ") + cudaGetErrorString(e));
        return TMC_CUDA_ERROR;
    }
    return TMC_OK;
}

int launched(tmc_status *st) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        put(st, TMC_CUDA_ERROR, std::string("CUDA error: ") + cudaGetErrorString(e));
        return TMC_CUDA_ERROR;
    }
    return TMC_OK;
}

}  // namespace
}  // namespace tmc

using namespace tmc;

extern "C" {

int tmc_b200_gemm_bf16(const uint16_t *A, const uint16_t *B, const float *bias, float *D, int32_t M, int32_t N,
                       int32_t K, void *stream, tmc_status *st) {
    put(st, TMC_OK, "");
    if (!D) {
        put(st, TMC_BAD_ARGUMENT, "NULL argument");
        return TMC_BAD_ARGUMENT;
    }
    const int dev = current_device();
    int *status = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        status = status_word(dev);
    }
    if (!status) {
        put(st, TMC_NO_DEVICE, "no usable CUDA device found");
        return TMC_NO_DEVICE;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaMemsetAsync(status, 0, sizeof(int), s);
    const int rc = launch_gemm(A, B, M, N, K, EpiF32{D, bias, N, 0}, stream, st);
    if (rc != TMC_OK) return rc;
    const cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        put(st, TMC_CUDA_ERROR, std::string("CUDA error in the tensor-core GEMM: ") + cudaGetErrorString(e));
        return TMC_CUDA_ERROR;
    }
    int h = 0;
    cudaMemcpy(&h, status, sizeof(int), cudaMemcpyDeviceToHost);
    if (h) {
        put(st, TMC_DEVICE_TIMEOUT, "a tensor-core wait gave up (mbarrier poll limit)");
        return TMC_DEVICE_TIMEOUT;
    }
    return TMC_OK;
}

int tmc_b200_probe_wait_timeout(int32_t device, uint32_t wait_limit, tmc_status *st) {
    put(st, TMC_OK, "");
    if (wait_limit < 1 || wait_limit > kGemmWaitLimit) {
        put(st, TMC_BAD_ARGUMENT, "wait_limit must be between 1 and the production limit");
        return TMC_BAD_ARGUMENT;
    }
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
        cudaGetLastError();
        put(st, TMC_NO_DEVICE, "no usable CUDA device found");
        return TMC_NO_DEVICE;
    }
    int saved = 0;
    cudaGetDevice(&saved);
    cudaSetDevice(device);
    // one 128 x 128 x 64 product whose producer issues no loads: the issuer's wait runs out
    void *buf = nullptr;
    const size_t a_bytes = 128 * 64 * 2, d_bytes = 128 * 128 * 4;
    if (cudaMalloc(&buf, 2 * a_bytes + d_bytes) != cudaSuccess) {
        cudaGetLastError();
        cudaSetDevice(saved);
        put(st, TMC_CUDA_ERROR, "CUDA error: cannot allocate the probe's operands");
        return TMC_CUDA_ERROR;
    }
    cudaMemset(buf, 0, 2 * a_bytes + d_bytes);
    unsigned char *b = static_cast<unsigned char *>(buf);
    int *status = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        status = status_word(device);
    }
    int rc = TMC_OK;
    if (!status) {
        put(st, TMC_NO_DEVICE, "no usable CUDA device found");
        rc = TMC_NO_DEVICE;
    } else {
        cudaMemset(status, 0, sizeof(int));
        rc = launch_gemm(b, b + a_bytes, 128, 128, 64, EpiF32{reinterpret_cast<float *>(b + 2 * a_bytes), nullptr, 128, 0},
                         nullptr, st, 1, wait_limit, 1);
        if (rc == TMC_OK) {
            const cudaError_t e = cudaDeviceSynchronize();
            int h = 0;
            if (e == cudaSuccess) cudaMemcpy(&h, status, sizeof(int), cudaMemcpyDeviceToHost);
            if (e != cudaSuccess) {
                put(st, TMC_CUDA_ERROR, std::string("CUDA error in the wait probe: ") + cudaGetErrorString(e));
                rc = TMC_CUDA_ERROR;
            } else if (h) {
                put(st, TMC_DEVICE_TIMEOUT, h == 1 ? "a tensor-core wait gave up (mbarrier poll limit)"
                                                   : "a tensor-core wait gave up and the CTA's own work did not drain");
                rc = TMC_DEVICE_TIMEOUT;
            }
            cudaMemset(status, 0, sizeof(int));
        }
    }
    cudaFree(buf);
    cudaSetDevice(saved);
    return rc;
}

int tmc_b200_nn_linear(const uint16_t *X, const uint16_t *W, const float *bias, float *Z, uint16_t *H, uint16_t *HT,
                       int32_t M, int32_t N, int32_t K, int32_t gelu_act, void *stream, tmc_status *st) {
    put(st, TMC_OK, "");
    if (!bias || (!Z && !H && !HT)) {
        put(st, TMC_BAD_ARGUMENT, "NULL argument");
        return TMC_BAD_ARGUMENT;
    }
    return launch_gemm(X, W, M, N, K,
                       EpiFwd{bias, Z, reinterpret_cast<__nv_bfloat16 *>(H), N, gelu_act,
                              reinterpret_cast<__nv_bfloat16 *>(HT), M},
                       stream, st);
}

int tmc_b200_nn_backward_data(const uint16_t *dZ, const uint16_t *WT, const float *Zprev, uint16_t *dX, uint16_t *dXT,
                              int32_t M, int32_t N, int32_t K, void *stream, tmc_status *st) {
    put(st, TMC_OK, "");
    if (!Zprev || !dX) {
        put(st, TMC_BAD_ARGUMENT, "NULL argument");
        return TMC_BAD_ARGUMENT;
    }
    return launch_gemm(dZ, WT, M, N, K,
                       EpiBwd{Zprev, reinterpret_cast<__nv_bfloat16 *>(dX), N, reinterpret_cast<__nv_bfloat16 *>(dXT), M},
                       stream, st);
}

int tmc_b200_nn_matmul_f32(const uint16_t *A, const uint16_t *B, float *D, int32_t M, int32_t N, int32_t K,
                           void *stream, tmc_status *st) {
    put(st, TMC_OK, "");
    if (!D) {
        put(st, TMC_BAD_ARGUMENT, "NULL argument");
        return TMC_BAD_ARGUMENT;
    }
    return launch_gemm(A, B, M, N, K, EpiF32{D, nullptr, N, 0}, stream, st);
}

int tmc_b200_nn_matmul_f32_splitk(const uint16_t *A, const uint16_t *B, float *D, float *work, int32_t M, int32_t N,
                                  int32_t K, int32_t splits, void *stream, tmc_status *st) {
    put(st, TMC_OK, "");
    if (!D || !work) {
        put(st, TMC_BAD_ARGUMENT, "NULL argument");
        return TMC_BAD_ARGUMENT;
    }
    const size_t mn = static_cast<size_t>(M) * N;
    const int rc = launch_gemm(A, B, M, N, K, EpiF32{work, nullptr, N, mn}, stream, st, splits);
    if (rc != TMC_OK) return rc;
    sum_splits_kernel<<<static_cast<unsigned>((mn + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        work, D, mn, splits);
    return launched(st);
}

int tmc_b200_nn_transpose(const uint16_t *X, uint16_t *Y, int32_t rows, int32_t cols, void *stream,
                          tmc_status *st) {
    put(st, TMC_OK, "");
    if (!X || !Y || rows < 1 || cols < 1) {
        put(st, TMC_BAD_ARGUMENT, "NULL argument or empty matrix");
        return TMC_BAD_ARGUMENT;
    }
    transpose_bf16_kernel<<<dim3((cols + 31) / 32, (rows + 31) / 32), dim3(32, 8), 0,
                            static_cast<cudaStream_t>(stream)>>>(reinterpret_cast<const __nv_bfloat16 *>(X),
                                                                 reinterpret_cast<__nv_bfloat16 *>(Y), rows, cols);
    return launched(st);
}

int tmc_b200_nn_colsum(const uint16_t *dZ, float *db, int32_t M, int32_t N, float *work, void *stream,
                       tmc_status *st) {
    put(st, TMC_OK, "");
    if (!dZ || !db || !work || M < 1 || N < 1) {
        put(st, TMC_BAD_ARGUMENT, "NULL argument or empty matrix");
        return TMC_BAD_ARGUMENT;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int groups = M < kColsumGroups ? M : kColsumGroups;
    colsum_partial_kernel<<<dim3((N + 127) / 128, groups), 128, 0, s>>>(reinterpret_cast<const __nv_bfloat16 *>(dZ),
                                                                      work, M, N);
    colsum_final_kernel<<<(N + 7) / 8, 256, 0, s>>>(work, db, N, groups);  // 8 columns (warps) per block
    return launched(st);
}

int32_t tmc_b200_nn_colsum_work(int32_t N) { return N < 1 ? 0 : kColsumGroups * N; }

int tmc_b200_nn_mse(const float *pred, const float *target, uint16_t *dZ, float *loss, int32_t M, int32_t T,
                    int32_t ld, float scale, void *stream, tmc_status *st) {
    put(st, TMC_OK, "");
    if (!pred || !target || !loss || M < 1 || T < 1 || ld < T) {
        put(st, TMC_BAD_ARGUMENT, "NULL argument or bad shape");
        return TMC_BAD_ARGUMENT;
    }
    const size_t n = static_cast<size_t>(M) * ld;
    const size_t blocks = std::min<size_t>((n + 255) / 256, 1184);  // at most 8 blocks per SM of a B200
    mse_kernel<<<static_cast<unsigned>(blocks), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        pred, target, reinterpret_cast<__nv_bfloat16 *>(dZ), loss, M, T, ld, scale);
    return launched(st);
}

int tmc_b200_nn_adam(float *w, const float *g, float *m, float *v, int32_t rows, int32_t cols, float lr_t,
                     const float *lr_dev, float b1, float b2, float eps, float weight_decay, uint16_t *wb, uint16_t *wt,
                     float *avg, float avg_beta, void *stream, tmc_status *st) {
    put(st, TMC_OK, "");
    if (!w || !g || !m || !v || rows < 1 || cols < 1) {
        put(st, TMC_BAD_ARGUMENT, "NULL argument or empty parameter");
        return TMC_BAD_ARGUMENT;
    }
    const size_t n = static_cast<size_t>(rows) * cols;
    adam_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        w, g, m, v, rows, cols, lr_t, lr_dev, b1, b2, eps, weight_decay, reinterpret_cast<__nv_bfloat16 *>(wb),
        reinterpret_cast<__nv_bfloat16 *>(wt), avg, avg_beta);
    return launched(st);
}

int32_t tmc_b200_nn_adam_plan(tmc_adam_tensor *tab, int32_t count) {
    if (!tab || count < 1) return -1;
    int64_t blocks = 0;
    for (int t = 0; t < count; ++t) {
        if (tab[t].rows < 1 || tab[t].cols < 1) return -1;
        tab[t].first_block = static_cast<int32_t>(blocks);
        blocks += (static_cast<int64_t>(tab[t].rows) * tab[t].cols + kAdamThreads - 1) / kAdamThreads;
        if (blocks > 0x7FFFFFFF) return -1;
    }
    return static_cast<int32_t>(blocks);
}

int tmc_b200_nn_adam_multi(const tmc_adam_tensor *tab, int32_t count, int32_t blocks, float lr_t, const float *lr_dev,
                           float b1, float b2, float eps, float avg_beta, void *stream, tmc_status *st) {
    put(st, TMC_OK, "");
    if (!tab || count < 1 || blocks < 1) {
        put(st, TMC_BAD_ARGUMENT, "NULL table, no tensors or no blocks (plan the table first)");
        return TMC_BAD_ARGUMENT;
    }
    adam_multi_kernel<<<static_cast<unsigned>(blocks), kAdamThreads, 0, static_cast<cudaStream_t>(stream)>>>(
        tab, count, lr_t, lr_dev, b1, b2, eps, avg_beta);
    return launched(st);
}

int tmc_b200_nn_ema(const float *w, float *avg, int64_t n, float beta, void *stream, tmc_status *st) {
    put(st, TMC_OK, "");
    if (!w || !avg || n < 1) {
        put(st, TMC_BAD_ARGUMENT, "NULL argument or empty parameter");
        return TMC_BAD_ARGUMENT;
    }
    ema_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        w, avg, static_cast<size_t>(n), beta);
    return launched(st);
}

int tmc_b200_nn_to_bf16(const float *w, int32_t rows, int32_t cols, uint16_t *wb, uint16_t *wt, void *stream,
                        tmc_status *st) {
    put(st, TMC_OK, "");
    if (!w || rows < 1 || cols < 1) {
        put(st, TMC_BAD_ARGUMENT, "NULL argument or empty parameter");
        return TMC_BAD_ARGUMENT;
    }
    const size_t n = static_cast<size_t>(rows) * cols;
    to_bf16_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        w, rows, cols, reinterpret_cast<__nv_bfloat16 *>(wb), reinterpret_cast<__nv_bfloat16 *>(wt));
    return launched(st);
}

int tmc_b200_nn_encode(const float *feats, const float *mean, const float *stdv, uint16_t *X, int32_t n, int32_t nf,
                       int32_t ld, void *stream, tmc_status *st) {
    put(st, TMC_OK, "");
    if (!feats || !mean || !stdv || !X || n < 1 || nf < 1 || ld < nf) {
        put(st, TMC_BAD_ARGUMENT, "NULL argument or bad shape");
        return TMC_BAD_ARGUMENT;
    }
    const size_t total = static_cast<size_t>(n) * ld;
    encode_kernel<<<static_cast<unsigned>((total + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        feats, mean, stdv, reinterpret_cast<__nv_bfloat16 *>(X), n, nf, ld);
    return launched(st);
}

int tmc_b200_nn_gate(const float *Z, int32_t members, int64_t member_stride, int32_t ld, const float *ymean,
                     const float *ystd, const float *areas, int32_t nbins, int32_t n, float threshold, float *rd_mean,
                     float *spread, uint8_t *route, void *stream, tmc_status *st) {
    put(st, TMC_OK, "");
    if (!Z || !ymean || !ystd || !areas || !route || members < 1 || n < 1 || nbins < 1 || ld < nbins) {
        put(st, TMC_BAD_ARGUMENT, "NULL argument or bad shape");
        return TMC_BAD_ARGUMENT;
    }
    gate_kernel<<<(n + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        Z, members, static_cast<size_t>(member_stride), ld, ymean, ystd, areas, nbins, n, threshold, rd_mean, spread,
        route);
    return launched(st);
}

int64_t tmc_b200_nn_packed_bytes(int32_t members) {
    return members < 1 ? 0 : static_cast<int64_t>(members) * kInferMemberBytes;
}

int tmc_b200_nn_pack(const uint16_t *const *weights, int32_t members, uint8_t *packed, void *stream,
                     tmc_status *st) {
    put(st, TMC_OK, "");
    if (!weights || !packed) {
        put(st, TMC_BAD_ARGUMENT, "NULL argument");
        return TMC_BAD_ARGUMENT;
    }
    if (members < 1 || members > kInferMaxMembers) {
        put(st, TMC_BAD_CONFIG, "the fused ensemble holds 1 to 8 members");
        return TMC_BAD_CONFIG;
    }
    PackParams P{};
    P.members = members;
    for (int i = 0; i < members * kInferLayers; ++i) {
        if (!weights[i] || reinterpret_cast<uintptr_t>(weights[i]) % 16 != 0) {
            put(st, TMC_BAD_ARGUMENT, "every weight matrix must be a non-NULL, 16-byte aligned device pointer");
            return TMC_BAD_ARGUMENT;
        }
        P.w[i] = reinterpret_cast<const __nv_bfloat16 *>(weights[i]);
    }
    const size_t units = static_cast<size_t>(members) * (kInferMemberBytes / 16);
    pack_kernel<<<static_cast<unsigned>((units + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(P, packed);
    return launched(st);
}

int tmc_b200_nn_ensemble_infer(const uint8_t *packed, const float *bias, int32_t members, const float *feats, int32_t n,
                               int32_t n_feat, const float *x_mean, const float *x_std, int32_t n_out,
                               const float *y_mean, const float *y_std, const float *areas, int32_t nbins,
                               float threshold, float *out, float *rd_mean, float *spread, uint8_t *route,
                               void *stream, tmc_status *st) {
    put(st, TMC_OK, "");
    if (!packed || !bias || !x_mean || !x_std || !y_mean || !y_std || (n > 0 && !feats) || (nbins > 0 && !areas)) {
        put(st, TMC_BAD_ARGUMENT, "NULL argument");
        return TMC_BAD_ARGUMENT;
    }
    if (members < 1 || members > kInferMaxMembers || n < 0 || n_feat < 1 || n_feat > kInferIn || n_out < 1 ||
        n_out > kInferOut || nbins < 0 || nbins > 64 || nbins > n_out) {
        put(st, TMC_BAD_CONFIG,
            "fused ensemble: 1-8 members, 1-64 input features, 1-128 outputs, 0-64 R_d bins among the outputs");
        return TMC_BAD_CONFIG;
    }
    if (n == 0) return TMC_OK;
    if (reinterpret_cast<uintptr_t>(packed) % 16 != 0) {
        put(st, TMC_BAD_ARGUMENT, "the packed weights must be 16-byte aligned");
        return TMC_BAD_ARGUMENT;
    }
    const int dev = current_device();
    int sms = 0;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        if (!status_word(dev) || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
            cudaGetLastError();
            put(st, TMC_NO_DEVICE, "no usable CUDA device found");
            return TMC_NO_DEVICE;
        }
        if (!g_infer_attr[dev]) {
            if (cudaFuncSetAttribute(ensemble_infer_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     InferSmem::bytes) != cudaSuccess)
                return launched(st);
            g_infer_attr[dev] = true;
        }
    }
    InferParams P{};
    P.packed = packed;
    P.bias = bias;
    P.feats = feats;
    P.x_mean = x_mean;
    P.x_std = x_std;
    P.y_mean = y_mean;
    P.y_std = y_std;
    P.areas = areas;
    P.out = out;
    P.rd_mean = rd_mean;
    P.spread = spread;
    P.route = route;
    P.n = n;
    P.n_feat = n_feat;
    P.n_out = n_out;
    P.nbins = nbins;
    P.members = members;
    P.threshold = threshold;
    P.status = g_status[dev];
    const int tiles = (n + 127) / 128;
    const int grid = tiles < sms ? tiles : sms;  // persistent: one CTA per SM (its shared memory allows no more)
    ensemble_infer_kernel<<<grid, kInferThreads, InferSmem::bytes, static_cast<cudaStream_t>(stream)>>>(P);
    return launched(st);
}

int tmc_b200_nn_status(int32_t clear) {
    const int dev = current_device();
    std::lock_guard<std::mutex> lock(g_mu);
    if (dev < 0 || dev >= 64 || !g_status[dev]) return 0;
    int h = 0;
    cudaMemcpy(&h, g_status[dev], sizeof(int), cudaMemcpyDeviceToHost);
    if (clear) cudaMemset(g_status[dev], 0, sizeof(int));
    return h;
}

}  // extern "C"
