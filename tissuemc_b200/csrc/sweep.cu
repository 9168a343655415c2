// Host side of the batched sweep (sweep_kernel.cuh): validation, the configuration sampler,
// device tables, one CUDA-graph-captured launch per sweep, and the launch-shape autotuner.

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/tissuemc_b200.h"
#include "engine_host.hpp"
#include "engine_internal.hpp"
#include "sweep_kernel.cuh"

namespace tmc {
// shared with the single-run loop in engine.cu
void sweep_block_to_layout(const uint64_t *src, int lmax, int nl, const tmc_sweep_options &o, uint64_t *dst);
}

namespace tmc {
namespace {

class SweepFail : public std::runtime_error {
  public:
    SweepFail(int code, const std::string &m) : std::runtime_error(m), code_(code) {}
    int code() const { return code_; }

  private:
    int code_;
};

#define SW_CUDA(call)                                                                                \
    do {                                                                                             \
        const cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                       \
            throw SweepFail(TMC_CUDA_ERROR, std::string("CUDA error at ") + __FILE__ + ":" +         \
                                                std::to_string(__LINE__) + ": " + cudaGetErrorString(e_)); \
    } while (0)

void put(tmc_status *st, int code, const std::string &m) {
    if (!st) return;
    st->code = code;
    std::snprintf(st->message, sizeof st->message, "%s", m.c_str());
}

// One configuration as a single run (for validation and for the single-run loop baseline).
tmc_run_spec as_run(const tmc_sweep_config &c, const tmc_sweep_options &o) {
    tmc_run_spec s;
    std::memset(&s, 0, sizeof s);
    s.photons = c.photons;
    s.dz = o.dz;
    s.dr = o.dr;
    s.nz = o.nz;
    s.nr = o.nr;
    s.na = o.na;
    s.n_above = c.n_above;
    s.n_below = c.n_below;
    s.num_layers = c.num_layers;
    for (int l = 0; l < c.num_layers && l < TMC_B200_MAX_LAYERS; ++l) s.layers[l] = c.layers[l];
    return s;
}

tmc_options as_options(const tmc_sweep_config &c, const tmc_sweep_options &o) {
    tmc_options r;
    tmc_b200_default_options(&r);
    r.seed = c.seed;
    r.batches = o.batches;
    r.rung = o.profiles ? 0 : 6;
    r.profiles = o.profiles;
    r.device = o.device;
    r.fast_math = o.fast_math;
    return r;
}

// Words between two configurations' tallies on the device: the block of one configuration, padded
// to 4 words above a multiple of 32. Measured on the 4096-configuration workload, the sweep's time
// depended on where its tally buffer landed (1.36-1.63 s with the unpadded 4294-word blocks, as
// allocations made before it moved the buffer), and with blocks of 4324 words it stayed within
// 1.36-1.39 s wherever it landed; the mechanism (how the configurations' hot lines spread over
// the L2 and DRAM) is not known. The padding is never copied out: results keep the run layout.
size_t device_stride(size_t words) { return (words + 27) / 32 * 32 + 4; }

struct SweepShape {
    int n, lmax;
    size_t stride;  // words per configuration
};

SweepShape validate_sweep(const tmc_sweep_config *cfgs, int n, const tmc_sweep_options &o) {
    if (n < 1) throw ConfigFailure("a sweep needs at least one configuration");
    if (o.threads_per_block < 0 || o.threads_per_block > 256 || o.threads_per_block % 32 != 0)
        throw ConfigFailure("threads_per_block must be a multiple of 32 in [32, 256] (0 = 256)");
    if (o.item_photons < 0) throw ConfigFailure("item_photons must be >= 0 (0 = 256)");
    if (o.tile_r < 0 || o.tile_z < 0 || (o.tile_r == 0) != (o.tile_z == 0))
        throw ConfigFailure("tile_r and tile_z must both be 0 (no tile) or both positive");
    if (o.tile_r > o.nr || o.tile_z > o.nz) throw ConfigFailure("the sweep's tile cannot exceed the grid");
    const int threads = o.threads_per_block > 0 ? o.threads_per_block : 256;
    if (static_cast<size_t>(threads / 32) * o.tile_r * o.tile_z * 8 > 32768)
        throw ConfigFailure("the sweep's tiles take more than 32 KB of shared memory per block");
    SweepShape sh{n, 1, 0};
    for (int i = 0; i < n; ++i) {
        try {
            validate_run(as_run(cfgs[i], o), as_options(cfgs[i], o));
        } catch (const ConfigFailure &e) {
            throw ConfigFailure("configuration " + std::to_string(i) + ": " + e.what());
        }
        sh.lmax = std::max(sh.lmax, cfgs[i].num_layers);
    }
    sh.stride = static_cast<size_t>(o.batches) * (4 + sh.lmax) + static_cast<size_t>(o.nr) * o.nz +
                2 * static_cast<size_t>(o.nr) * o.na;
    if (static_cast<double>(device_stride(sh.stride)) * n >= 2147483648.0)
        throw ConfigFailure("the sweep's tallies exceed 2^31 words (fewer configurations or bins)");
    return sh;
}

// ------------------------------------------------------------------------- host Philox
// Philox4x32-10 (Salmon et al. 2011) for drawing the sweep's configurations on the host.
void philox_host(uint32_t c[4], uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = static_cast<uint64_t>(0xD2511F53u) * c[0];
        const uint64_t p1 = static_cast<uint64_t>(0xCD9E8D57u) * c[2];
        const uint32_t n0 = static_cast<uint32_t>(p1 >> 32) ^ c[1] ^ k0;
        const uint32_t n2 = static_cast<uint32_t>(p0 >> 32) ^ c[3] ^ k1;
        c[0] = n0;
        c[1] = static_cast<uint32_t>(p1);
        c[2] = n2;
        c[3] = static_cast<uint32_t>(p0);
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

struct ConfigDraws {
    uint64_t seed;
    uint32_t cfg, blk;
    uint32_t buf[4];
    int used = 4;
    double next() {  // uniform on (0, 1) from 32 bits
        if (used == 4) {
            buf[0] = cfg;
            buf[1] = 0x7377u;  // a stream tag that keeps these draws apart from photon streams
            buf[2] = blk++;
            buf[3] = 0u;
            philox_host(buf, static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 32));
            used = 0;
        }
        return (static_cast<double>(buf[used++]) + 0.5) * 0x1p-32;
    }
};

// ------------------------------------------------------------------------- the captured sweep
struct SweepGraph {
    int device = -1;
    tmc_sweep_options opt{};
    int cap_cfg = 0, lmax = 0;
    size_t stride = 0;
    int threads = 256, grid = 0;
    size_t smem = 0;
    cudaStream_t stream = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    unsigned char *d_blob = nullptr, *h_blob = nullptr;
    size_t blob_bytes = 0, off_cfg = 0, off_prefix = 0, off_layers = 0;
    unsigned long long *d_tally = nullptr;
    unsigned int *d_counter = nullptr;
    double *d_summary = nullptr, *h_summary = nullptr;
    std::vector<int> order;  // table slot -> the caller's configuration (longest photons first)

    ~SweepGraph() {
        if (device >= 0) cudaSetDevice(device);
        if (exec) cudaGraphExecDestroy(exec);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (stream) cudaStreamDestroy(stream);
        cudaFree(d_blob);
        cudaFree(d_tally);
        cudaFree(d_counter);
        cudaFree(d_summary);
        cudaFreeHost(h_blob);
        cudaFreeHost(h_summary);
    }
};

size_t align_up(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }


bool same_shape(const tmc_sweep_options &a, const tmc_sweep_options &b) {
    return a.dz == b.dz && a.dr == b.dr && a.nz == b.nz && a.nr == b.nr && a.na == b.na &&
           a.batches == b.batches && a.fast_math == b.fast_math && a.profiles == b.profiles &&
           a.device == b.device && a.threads_per_block == b.threads_per_block && a.tile_r == b.tile_r &&
           a.tile_z == b.tile_z;
}

// Build (allocate, capture, instantiate) a sweep graph for up to cap configurations with up to
// lmax layers each: copy the tables in, zero tallies and the item counter, run the sweep kernel
// between two timing events, summarise, copy the summaries out.
std::unique_ptr<SweepGraph> build_graph(int cap, int lmax, const tmc_sweep_options &o) {
    auto g = std::make_unique<SweepGraph>();
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0 || o.device < 0 || o.device >= n) {
        cudaGetLastError();
        throw SweepFail(TMC_NO_DEVICE, "no usable CUDA device found");
    }
    SW_CUDA(cudaSetDevice(o.device));
    g->device = o.device;
    g->opt = o;
    g->cap_cfg = cap;
    g->lmax = lmax;
    g->stride = device_stride(static_cast<size_t>(o.batches) * (4 + lmax) + static_cast<size_t>(o.nr) * o.nz +
                              2 * static_cast<size_t>(o.nr) * o.na);
    g->threads = o.threads_per_block > 0 ? o.threads_per_block : 256;
    // per lane: the random-word ring (kRingWords words) and the Philox key schedule (5 x 16 bytes);
    // per warp: the optional tile of A(r,z)
    g->smem = (4 * kRingWords + 80) * static_cast<size_t>(g->threads) +
              static_cast<size_t>(g->threads / 32) * o.tile_r * o.tile_z * 8;
    cudaDeviceProp prop;
    SW_CUDA(cudaGetDeviceProperties(&prop, o.device));
    // the kernel for these options: fast or exact math, with or without the per-warp tile, or the
    // kernel of totals only (no profile tallies)
    const bool tile = o.profiles && o.tile_r > 0;
    const void *kern = !o.profiles ? (o.fast_math ? reinterpret_cast<const void *>(sweep_kernel_totals<1>)
                                                  : reinterpret_cast<const void *>(sweep_kernel_totals<0>))
                       : o.fast_math ? (tile ? reinterpret_cast<const void *>(sweep_kernel<1, true>)
                                             : reinterpret_cast<const void *>(sweep_kernel<1, false>))
                                     : (tile ? reinterpret_cast<const void *>(sweep_kernel<0, true>)
                                             : reinterpret_cast<const void *>(sweep_kernel<0, false>));
    SW_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(g->smem)));
    int bps = 0;
    SW_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, g->threads, g->smem));
    g->grid = prop.multiProcessorCount * std::max(1, bps);

    g->off_cfg = align_up(sizeof(SweepHeader));
    g->off_prefix = g->off_cfg + align_up(sizeof(SweepConfigC) * cap);
    g->off_layers = g->off_prefix + align_up(sizeof(uint32_t) * (cap + 1));
    g->blob_bytes = g->off_layers + align_up(sizeof(LayerC) * static_cast<size_t>(cap) * lmax);
    SW_CUDA(cudaMalloc(&g->d_blob, g->blob_bytes));
    SW_CUDA(cudaMallocHost(&g->h_blob, g->blob_bytes));
    SW_CUDA(cudaMalloc(&g->d_tally, g->stride * cap * 8));
    SW_CUDA(cudaMalloc(&g->d_counter, 256));
    const size_t sum_words = static_cast<size_t>(cap) * (o.nr + 3);
    SW_CUDA(cudaMalloc(&g->d_summary, sum_words * 8));
    SW_CUDA(cudaMallocHost(&g->h_summary, sum_words * 8));
    SW_CUDA(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
    SW_CUDA(cudaEventCreate(&g->e0));
    SW_CUDA(cudaEventCreate(&g->e1));

    SweepParams P{};
    P.hdr = reinterpret_cast<const SweepHeader *>(g->d_blob);
    P.cfgs = reinterpret_cast<const SweepConfigC *>(g->d_blob + g->off_cfg);
    P.prefix = reinterpret_cast<const uint32_t *>(g->d_blob + g->off_prefix);
    P.layers = reinterpret_cast<const LayerC *>(g->d_blob + g->off_layers);
    P.item_counter = g->d_counter;
    P.tally = g->d_tally;
    P.stride = static_cast<int>(g->stride);
    P.nb = o.batches;
    P.lmax = lmax;
    P.nz = o.nz;
    P.nr = o.nr;
    P.na = o.na;
    P.dz = static_cast<float>(o.dz);
    P.dr = static_cast<float>(o.dr);
    P.da = static_cast<float>(0.5 * 3.14159265358979323846 / o.na);
    P.inv_dz = 1.0f / P.dz;
    P.inv_dr = 1.0f / P.dr;
    P.inv_da = 1.0f / P.da;
    P.profiles = o.profiles ? 1 : 0;
    P.step_cap = 2000000000u;
    P.threads = static_cast<uint32_t>(g->threads);
    P.tile_r = o.profiles ? o.tile_r : 0;
    P.tile_z = o.profiles ? o.tile_z : 0;

    cudaGraph_t graph = nullptr;
    SW_CUDA(cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeThreadLocal));
    try {
        SW_CUDA(cudaMemcpyAsync(g->d_blob, g->h_blob, g->blob_bytes, cudaMemcpyHostToDevice, g->stream));
        SW_CUDA(cudaMemsetAsync(g->d_tally, 0, g->stride * cap * 8, g->stream));
        SW_CUDA(cudaMemsetAsync(g->d_counter, 0, 256, g->stream));
        SW_CUDA(cudaEventRecordWithFlags(g->e0, g->stream, cudaEventRecordExternal));
        void *args[] = {&P};
        SW_CUDA(cudaLaunchKernel(kern, dim3(g->grid), dim3(g->threads), args, g->smem, g->stream));
        SW_CUDA(cudaGetLastError());
        SW_CUDA(cudaEventRecordWithFlags(g->e1, g->stream, cudaEventRecordExternal));
        const int warps_per_block = 8;
        sweep_finalize_kernel<<<(cap + warps_per_block - 1) / warps_per_block, 32 * warps_per_block, 0, g->stream>>>(
            P.cfgs, g->d_tally, cap, P.stride, o.batches, lmax, o.nz, o.nr, o.na, g->d_summary);
        SW_CUDA(cudaGetLastError());
        SW_CUDA(cudaMemcpyAsync(g->h_summary, g->d_summary, sum_words * 8, cudaMemcpyDeviceToHost, g->stream));
    } catch (...) {
        cudaStreamEndCapture(g->stream, &graph);
        if (graph) cudaGraphDestroy(graph);
        throw;
    }
    SW_CUDA(cudaStreamEndCapture(g->stream, &graph));
    const cudaError_t ie = cudaGraphInstantiate(&g->exec, graph, 0);
    cudaGraphDestroy(graph);
    SW_CUDA(ie);
    return g;
}

// Steps a photon of this configuration is expected to take, for ordering only: the smaller of the
// interactions until roulette (the weight falls below 1e-4 after about ln(1e4) mu_t / mu_a
// interactions) and the scatterings a diffusing photon needs to cross the stack (about
// (tau' d)^2 mu_s / mu_s', tau' = mu_a + mu_s'), combined harmonically, with the stack's
// thickness-weighted optics. Ranks the sweep distribution's configurations by their measured
// mean steps per photon with a rank correlation of 0.99.
double photon_cost(const tmc_sweep_config &c) {
    double dt = 0.0, mua = 0.0, mus = 0.0, g = 0.0;
    for (int l = 0; l < c.num_layers; ++l) {
        const tmc_layer &y = c.layers[l];
        dt += y.d;
        mua += y.mua * y.d;
        mus += y.mus * y.d;
        g += y.g * y.d;
    }
    mua /= dt;
    mus /= dt;
    g /= dt;
    const double mut = mua + mus, musp = std::max(mus * (1.0 - g), 1e-12);
    const double tau = dt * (mua + musp);
    const double cross = tau * tau * mus / musp + mut * dt;
    return 1.0 / (mua / (9.21 * mut) + 1.0 / cross);
}

// Fill the pinned table blob for these configurations; returns the number of items. The table
// holds them longest photons first (g.order maps a slot back to the caller's index), and the
// items are taken in kSweepBands bands, so the long photons start early.
constexpr uint32_t kSweepBands = 16;

uint32_t fill_blob(SweepGraph &g, const tmc_sweep_config *cfgs, int n) {
    const tmc_sweep_options &o = g.opt;
    const uint32_t item = static_cast<uint32_t>(o.item_photons > 0 ? o.item_photons : 256);
    auto *cf = reinterpret_cast<SweepConfigC *>(g.h_blob + g.off_cfg);
    auto *prefix = reinterpret_cast<uint32_t *>(g.h_blob + g.off_prefix);
    auto *layers = reinterpret_cast<LayerC *>(g.h_blob + g.off_layers);
    std::vector<double> cost(static_cast<size_t>(n));
    g.order.resize(static_cast<size_t>(n));
    for (int c = 0; c < n; ++c) {
        cost[c] = photon_cost(cfgs[c]);
        g.order[c] = c;
    }
    std::stable_sort(g.order.begin(), g.order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
    uint64_t total = 0;
    int lbase = 0;
    for (int slot = 0; slot < n; ++slot) {
        const tmc_sweep_config &src = cfgs[g.order[slot]];
        const tmc_run_spec spec = as_run(src, o);
        SweepConfigC &k = cf[slot];
        k = SweepConfigC{};
        const uint32_t ph = static_cast<uint32_t>(src.photons);
        const uint32_t nb = static_cast<uint32_t>(o.batches);
        k.photons = ph;
        k.plan_base = ph / nb;
        k.plan_extra = ph % nb;
        k.plan_bnd = k.plan_extra * (k.plan_base + 1u);
        k.k0 = static_cast<uint32_t>(src.seed);
        k.k1 = static_cast<uint32_t>(src.seed >> 32);
        k.launch_w = launch_weight(spec);
        k.nl = spec.num_layers;
        k.layer_base = lbase;
        fill_layers(spec, layers + lbase);
        lbase += spec.num_layers;
        prefix[slot] = static_cast<uint32_t>(total);
        total += (ph + item - 1) / item;
    }
    if (total >= 0xFFFFFFFFull) throw ConfigFailure("too many work items; raise item_photons");
    prefix[n] = static_cast<uint32_t>(total);
    const SweepHeader h{static_cast<uint32_t>(n), item, sweep_order(static_cast<uint32_t>(total), kSweepBands)};
    std::memcpy(g.h_blob, &h, sizeof h);
    return h.order.total;
}

std::mutex g_sweep_mu;
std::unique_ptr<SweepGraph> g_cached[64];

SweepGraph &graph_for(int n, int lmax, const tmc_sweep_options &o) {
    if (o.device < 0 || o.device >= 64) throw ConfigFailure("device ordinal out of range");
    std::unique_ptr<SweepGraph> &slot = g_cached[o.device];
    if (!slot || slot->cap_cfg < n || slot->lmax < lmax || !same_shape(slot->opt, o)) {
        const bool keep = slot && same_shape(slot->opt, o);
        const int cap = keep ? std::max(n, slot->cap_cfg) : n;
        const int lm = keep ? std::max(lmax, slot->lmax) : lmax;
        slot.reset();  // free the old graph's memory before allocating the new one
        slot = build_graph(cap, lm, o);
    }
    slot->opt.item_photons = o.item_photons;
    return *slot;
}

// Copy one configuration's tallies from a block with lmax layer slots per batch row into a block
// with nl slots per row (nl <= lmax: the single-run layout of a configuration with nl layers).
void sweep_to_run_layout(const uint64_t *src, int lmax, int nl, const tmc_sweep_options &o, uint64_t *dst) {
    const size_t profile = static_cast<size_t>(o.nr) * o.nz + 2 * static_cast<size_t>(o.nr) * o.na;
    for (int b = 0; b < o.batches; ++b)
        for (int i = 0; i < 4 + nl; ++i) dst[static_cast<size_t>(b) * (4 + nl) + i] = src[static_cast<size_t>(b) * (4 + lmax) + i];
    std::memcpy(dst + static_cast<size_t>(o.batches) * (4 + nl), src + static_cast<size_t>(o.batches) * (4 + lmax),
                profile * 8);
}

}  // namespace

void sweep_block_to_layout(const uint64_t *src, int lmax, int nl, const tmc_sweep_options &o, uint64_t *dst) {
    sweep_to_run_layout(src, lmax, nl, o, dst);
}

}  // namespace tmc

using namespace tmc;

extern "C" {

void tmc_b200_sweep_default_options(tmc_sweep_options *o) {
    if (!o) return;
    std::memset(o, 0, sizeof *o);
    o->dz = 0.01;
    o->dr = 0.01;
    o->nz = 64;
    o->nr = 64;
    o->na = 1;
    o->batches = 10;
    o->fast_math = 1;
    o->profiles = 1;
    o->device = 0;
    o->threads_per_block = 256;
    o->item_photons = 256;
}

int tmc_b200_sweep_sample(uint64_t master_seed, int32_t n, tmc_sweep_config *out, tmc_status *st) {
    put(st, TMC_OK, "");
    if (!out || n < 0) {
        put(st, TMC_BAD_ARGUMENT, "NULL argument or negative count");
        return TMC_BAD_ARGUMENT;
    }
    for (int c = 0; c < n; ++c) {
        ConfigDraws d{master_seed, static_cast<uint32_t>(c), 0u, {0, 0, 0, 0}, 4};
        tmc_sweep_config &k = out[c];
        std::memset(&k, 0, sizeof k);
        k.num_layers = 1 + std::min(2, static_cast<int>(d.next() * 3.0));
        const double nidx = 1.33 + 0.17 * d.next();  // one index for every layer of a configuration
        k.n_above = 1.0;
        k.n_below = 1.0;
        for (int l = 0; l < k.num_layers; ++l) {
            const double mua = std::pow(10.0, -2.0 + 3.0 * d.next());           // [0.01, 10] /cm
            const double musp = std::pow(10.0, std::log10(50.0) * d.next());   // [1, 50] /cm
            const double g = 0.7 + 0.25 * d.next();                             // [0.7, 0.95]
            const double dd = std::pow(10.0, -2.0 + 2.0 * d.next());            // [0.01, 1] cm
            k.layers[l] = tmc_layer{nidx, mua, musp / (1.0 - g), g, dd};
        }
        k.photons = static_cast<uint64_t>(std::floor(std::pow(10.0, 4.0 + 2.0 * d.next())));  // [1e4, 1e6]
        const uint64_t lo = static_cast<uint64_t>(d.next() * 4294967296.0);
        const uint64_t hi = static_cast<uint64_t>(d.next() * 4294967296.0);
        k.seed = (hi << 32) | lo;
    }
    return TMC_OK;
}

int tmc_b200_sweep_costs(const tmc_sweep_config *cfgs, int32_t n, double *cost, tmc_status *st) {
    put(st, TMC_OK, "");
    if (!cfgs || !cost || n < 0) {
        put(st, TMC_BAD_ARGUMENT, "NULL argument or negative count");
        return TMC_BAD_ARGUMENT;
    }
    for (int c = 0; c < n; ++c) {
        if (cfgs[c].num_layers < 1 || cfgs[c].num_layers > TMC_B200_MAX_LAYERS) {
            put(st, TMC_BAD_CONFIG, "configuration " + std::to_string(c) + ": 1 to 16 layers are needed");
            return TMC_BAD_CONFIG;
        }
        cost[c] = photon_cost(cfgs[c]);
    }
    return TMC_OK;
}

int tmc_b200_sweep_sizes(const tmc_sweep_config *cfgs, int32_t n, const tmc_sweep_options *opt,
                         tmc_sweep_sizes *sz, tmc_status *st) {
    put(st, TMC_OK, "");
    if (!cfgs || !opt || !sz) {
        put(st, TMC_BAD_ARGUMENT, "NULL argument");
        return TMC_BAD_ARGUMENT;
    }
    try {
        const SweepShape sh = validate_sweep(cfgs, n, *opt);
        sz->words_per_config = sh.stride;
        sz->summary_per_config = static_cast<uint64_t>(opt->nr) + 3;
        sz->max_layers = sh.lmax;
        return TMC_OK;
    } catch (const ConfigFailure &e) {
        put(st, TMC_BAD_CONFIG, e.what());
        return TMC_BAD_CONFIG;
    }
}

int tmc_b200_sweep_run(const tmc_sweep_config *cfgs, int32_t n, const tmc_sweep_options *opt, uint64_t *raw,
                       double *summary, double *kernel_seconds, tmc_status *st) {
    put(st, TMC_OK, "");
    if (!cfgs || !opt) {
        put(st, TMC_BAD_ARGUMENT, "NULL argument");
        return TMC_BAD_ARGUMENT;
    }
    std::lock_guard<std::mutex> lock(g_sweep_mu);
    try {
        const SweepShape sh = validate_sweep(cfgs, n, *opt);
        SweepGraph &g = graph_for(n, sh.lmax, *opt);
        fill_blob(g, cfgs, n);
        SW_CUDA(cudaSetDevice(g.device));
        SW_CUDA(cudaGraphLaunch(g.exec, g.stream));
        SW_CUDA(cudaStreamSynchronize(g.stream));
        float ms = 0.f;
        SW_CUDA(cudaEventElapsedTime(&ms, g.e0, g.e1));
        if (kernel_seconds) *kernel_seconds = static_cast<double>(ms) / 1000.0;
        // results come back in the caller's order (the table holds configurations by photon cost)
        const size_t sw = static_cast<size_t>(opt->nr) + 3;
        if (summary)
            for (int slot = 0; slot < n; ++slot)
                std::memcpy(summary + static_cast<size_t>(g.order[slot]) * sw, g.h_summary + slot * sw, sw * 8);
        if (raw) {
            // every configuration's block, in the layout of this call (sh.lmax layer slots per row)
            std::vector<uint64_t> all(g.stride * n);
            SW_CUDA(cudaMemcpy(all.data(), g.d_tally, g.stride * n * 8, cudaMemcpyDeviceToHost));
            for (int slot = 0; slot < n; ++slot) {
                const uint64_t *src = all.data() + static_cast<size_t>(slot) * g.stride;
                uint64_t *dst = raw + static_cast<size_t>(g.order[slot]) * sh.stride;
                if (g.lmax == sh.lmax) std::memcpy(dst, src, sh.stride * 8);  // any padding stays behind
                else sweep_to_run_layout(src, g.lmax, sh.lmax, *opt, dst);
            }
        }
        return TMC_OK;
    } catch (const ConfigFailure &e) {
        put(st, TMC_BAD_CONFIG, e.what());
        return TMC_BAD_CONFIG;
    } catch (const SweepFail &e) {
        put(st, e.code(), e.what());
        return e.code();
    } catch (const std::exception &e) {
        put(st, TMC_CUDA_ERROR, e.what());
        return TMC_CUDA_ERROR;
    }
}

int tmc_b200_sweep_run_loop(const tmc_sweep_config *cfgs, int32_t n, const tmc_sweep_options *opt, uint64_t *raw,
                            double *seconds, tmc_status *st) {
    put(st, TMC_OK, "");
    if (!cfgs || !opt) {
        put(st, TMC_BAD_ARGUMENT, "NULL argument");
        return TMC_BAD_ARGUMENT;
    }
    try {
        const SweepShape sh = validate_sweep(cfgs, n, *opt);
        std::vector<tmc_run_spec> specs(n);
        std::vector<tmc_options> opts(n);
        for (int c = 0; c < n; ++c) {
            specs[c] = as_run(cfgs[c], *opt);
            opts[c] = as_options(cfgs[c], *opt);
        }
        std::vector<uint64_t> all;
        std::vector<size_t> offsets;
        const double secs = run_single_loop(specs.data(), opts.data(), n, raw ? &all : nullptr, &offsets);
        if (seconds) *seconds = secs;
        if (raw) {
            // each run's own layout (nl layer slots per batch row) widened to the sweep's lmax
            for (int c = 0; c < n; ++c) {
                const uint64_t *src = all.data() + offsets[c];
                uint64_t *dst = raw + static_cast<size_t>(c) * sh.stride;
                std::memset(dst, 0, sh.stride * 8);
                const int nl = cfgs[c].num_layers;
                for (int b = 0; b < opt->batches; ++b)
                    for (int i = 0; i < 4 + nl; ++i)
                        dst[static_cast<size_t>(b) * (4 + sh.lmax) + i] = src[static_cast<size_t>(b) * (4 + nl) + i];
                const size_t profile = static_cast<size_t>(opt->nr) * opt->nz + 2 * static_cast<size_t>(opt->nr) * opt->na;
                std::memcpy(dst + static_cast<size_t>(opt->batches) * (4 + sh.lmax),
                            src + static_cast<size_t>(opt->batches) * (4 + nl), profile * 8);
            }
        }
        return TMC_OK;
    } catch (const ConfigFailure &e) {
        put(st, TMC_BAD_CONFIG, e.what());
        return TMC_BAD_CONFIG;
    } catch (const std::exception &e) {
        put(st, TMC_CUDA_ERROR, e.what());
        return TMC_CUDA_ERROR;
    }
}

int tmc_b200_sweep_autotune(const tmc_sweep_config *cfgs, int32_t n, tmc_sweep_options *opt, double *best_seconds,
                            tmc_status *st) {
    put(st, TMC_OK, "");
    if (!cfgs || !opt) {
        put(st, TMC_BAD_ARGUMENT, "NULL argument");
        return TMC_BAD_ARGUMENT;
    }
    // Candidates: block size x photons per work item, timed on this sweep (second of two runs). The
    // caller's options are timed first and are replaced only by a candidate at least 1.5 % faster
    // (the run-to-run spread of a sweep is a few tenths of a percent).
    auto time_of = [&](tmc_sweep_options &o, double &secs) {
        for (int rep = 0; rep < 2; ++rep) {
            const int rc = tmc_b200_sweep_run(cfgs, n, &o, nullptr, nullptr, &secs, st);
            if (rc != TMC_OK) return rc;
        }
        return static_cast<int>(TMC_OK);
    };
    tmc_sweep_options best = *opt;
    double best_t = 1e300;
    if (const int rc = time_of(best, best_t); rc != TMC_OK) return rc;
    const int threads[] = {128, 256};
    const int items[] = {64, 256, 1024};
    for (int t : threads) {
        for (int it : items) {
            tmc_sweep_options o = best;
            o.threads_per_block = t;
            o.item_photons = it;
            if (o.threads_per_block == best.threads_per_block && o.item_photons == best.item_photons) continue;
            double secs = 0;
            if (const int rc = time_of(o, secs); rc != TMC_OK) return rc;
            if (secs < best_t * 0.985) {
                best_t = secs;
                best = o;
            }
        }
    }
    // then the per-warp tile of A(r,z), with the best launch shape
    const int tiles[][2] = {{8, 8}, {16, 16}, {16, 32}};
    for (const auto &tl : tiles) {
        tmc_sweep_options o = best;
        o.tile_r = std::min(tl[0], o.nr);
        o.tile_z = std::min(tl[1], o.nz);
        const int th = o.threads_per_block > 0 ? o.threads_per_block : 256;
        if (static_cast<size_t>(th / 32) * o.tile_r * o.tile_z * 8 > 32768) continue;
        double secs = 0;
        for (int rep = 0; rep < 2; ++rep) {
            const int rc = tmc_b200_sweep_run(cfgs, n, &o, nullptr, nullptr, &secs, st);
            if (rc != TMC_OK) return rc;
        }
        if (secs < best_t * 0.985) {
            best_t = secs;
            best = o;
        }
    }
    *opt = best;
    if (best_seconds) *best_seconds = best_t;
    return TMC_OK;
}

}  // extern "C"
