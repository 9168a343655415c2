// Physics probe (tmc_b200_probe_physics): the walk's own device functions — the free-path length,
// the Henyey-Greenstein sampler and the direction rotation of walk_step.cuh — run in isolation on
// many Philox streams, so that tests can check them the way TissueMC's unit tests check its CPU
// physics (tests/cpp/test_physics.cpp:91-160): the sampler's first two moments, the unit norm of the
// direction over millions of consecutive scatterings, and the mean free path.

#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/tissuemc_b200.h"
#include "engine_internal.hpp"
#include "walk_step.cuh"

namespace tmc {
namespace {

constexpr int kProbeThreads = 256, kProbeBlocks = 296;

// Uniform draws of one thread's stream (seed, thread): four words per Philox block.
struct ProbeRng {
    uint32_t id, blk, k0, k1, buf[4];
    int used;
    __device__ float next() {
        if (used == 4) {
            philox4x32_10(id, 0u, blk++, k0, k1, buf[0], buf[1], buf[2], buf[3]);
            used = 0;
        }
        return unit_open(buf[used++]);
    }
};

// what 0: Henyey-Greenstein cosines: out[0] += cos, out[1] += cos^2, out[2] = min, out[3] = max.
// what 1: consecutive rotations of one direction per thread: out[0] = worst |norm - 1|.
// what 2: free paths: out[0] += s, out[1] += s^2.
template <int FAST>
__global__ void probe_kernel(int what, Hot h, uint64_t seed, long long per_thread, double *out) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    ProbeRng rng{tid, 0u, static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 32), {0u, 0u, 0u, 0u}, 4};
    double s1 = 0.0, s2 = 0.0;
    float lo = 2.0f, hi = -2.0f, worst = 0.0f;
    float2 uxy = make_float2(0.0f, 0.0f);
    float uz = 1.0f;
    for (long long i = 0; i < per_thread; ++i) {
        if (what == 0) {
            const float c = hg_cos<FAST>(h, rng.next());
            s1 += c;
            s2 += static_cast<double>(c) * c;
            lo = fminf(lo, c);
            hi = fmaxf(hi, c);
        } else if (what == 1) {
            const float ct = hg_cos<FAST>(h, rng.next());
            rotate<FAST>(uxy, uz, ct, rng.next());
            const double ux = uxy.x, uy = uxy.y;
            const float n = sqrtf(static_cast<float>(ux * ux + uy * uy + static_cast<double>(uz) * uz));
            worst = fmaxf(worst, fabsf(n - 1.0f));
        } else {
            const float s = step_length<FAST>(h, rng.next());
            s1 += s;
            s2 += static_cast<double>(s) * s;
        }
    }
    if (what == 0) {
        atomicAdd(&out[0], s1);
        atomicAdd(&out[1], s2);
        // min / max of floats in [-1, 1] through the order-preserving integer view of their
        // shifted values (c + 2 > 0)
        atomicMin(reinterpret_cast<unsigned long long *>(&out[2]),
                  static_cast<unsigned long long>(__double_as_longlong(static_cast<double>(lo) + 2.0)));
        atomicMax(reinterpret_cast<unsigned long long *>(&out[3]),
                  static_cast<unsigned long long>(__double_as_longlong(static_cast<double>(hi) + 2.0)));
    } else if (what == 1) {
        atomicMax(reinterpret_cast<unsigned long long *>(&out[0]),
                  static_cast<unsigned long long>(__double_as_longlong(static_cast<double>(worst))));
    } else {
        atomicAdd(&out[0], s1);
        atomicAdd(&out[1], s2);
    }
}

}  // namespace
}  // namespace tmc

using namespace tmc;

extern "C" int tmc_b200_probe_physics(int32_t what, double g, double mu_t, int64_t samples, uint64_t seed,
                                      int32_t fast_math, int32_t device, double *out, tmc_status *st) {
    auto status = [&](int code, const std::string &m) {
        if (st) {
            st->code = code;
            std::snprintf(st->message, sizeof st->message, "%s", m.c_str());
        }
        return code;
    };
    status(TMC_OK, "");
    if (!out) return status(TMC_BAD_ARGUMENT, "NULL argument");
    if (what < 0 || what > 2 || !(g > -1.0 && g < 1.0) || !(mu_t > 0.0) || samples < 1)
        return status(TMC_BAD_CONFIG, "probe: what in 0..2, -1 < g < 1, mu_t > 0, samples >= 1");
    if (cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        return status(TMC_NO_DEVICE, "no usable CUDA device found");
    }
    // one layer with these optics, its constants computed as for a run
    tmc_run_spec spec;
    std::memset(&spec, 0, sizeof spec);
    spec.photons = 1;
    spec.dz = spec.dr = 0.01;
    spec.nz = spec.nr = spec.na = 1;
    spec.n_above = spec.n_below = 1.0;
    spec.num_layers = 1;
    spec.layers[0] = tmc_layer{1.0, 0.1 * mu_t, 0.9 * mu_t, g, 1.0};
    LayerC L[1];
    fill_layers(spec, L);
    Hot h;
    h.mua = L[0].mua;
    h.mut = L[0].mut;
    h.inv_mut = L[0].inv_mut;
    h.absorb = L[0].absorb;
    h.z0 = L[0].z0;
    h.z1 = L[0].z1;
    h.g = L[0].g;
    h.hg_a = L[0].hg_a;
    h.hg_b = L[0].hg_b;
    h.hg_c = L[0].hg_c;
    h.hg_d = L[0].hg_d;
    h.inv_2g = L[0].inv_2g;
    // rotations chain within a thread (the norm's drift over consecutive scatterings is the point):
    // one warp, so that each of its 32 directions sees samples / 32 consecutive rotations
    const int blocks = what == 1 ? 1 : kProbeBlocks, block = what == 1 ? 32 : kProbeThreads;
    const long long threads = static_cast<long long>(block) * blocks;
    const long long per_thread = (samples + threads - 1) / threads;
    double init[4] = {0.0, 0.0, 0.0, 0.0};
    if (what == 0) {  // min and max start at the ends of the shifted range [1, 3]
        init[2] = 3.5;
        init[3] = 0.5;
    }
    double *d_out = nullptr;
    // a probe is a diagnostic: it owns a small device buffer for the duration of the call
    if (cudaMalloc(&d_out, sizeof init) != cudaSuccess ||
        cudaMemcpy(d_out, init, sizeof init, cudaMemcpyHostToDevice) != cudaSuccess) {
        const std::string m = cudaGetErrorString(cudaGetLastError());
        if (d_out) cudaFree(d_out);
        return status(TMC_CUDA_ERROR, "CUDA error in the physics probe: " + m);
    }
    if (fast_math)
        probe_kernel<1><<<blocks, block>>>(what, h, seed, per_thread, d_out);
    else
        probe_kernel<0><<<blocks, block>>>(what, h, seed, per_thread, d_out);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(init, d_out, sizeof init, cudaMemcpyDeviceToHost);
    cudaFree(d_out);
    if (e != cudaSuccess) return status(TMC_CUDA_ERROR, std::string("CUDA error in the physics probe: ") + cudaGetErrorString(e));
    const double n = static_cast<double>(per_thread * threads);
    out[4] = n;
    if (what == 0) {
        out[0] = init[0];
        out[1] = init[1];
        out[2] = init[2] - 2.0;
        out[3] = init[3] - 2.0;
    } else {
        out[0] = init[0];
        out[1] = init[1];
        out[2] = out[3] = 0.0;
    }
    return TMC_OK;
}
