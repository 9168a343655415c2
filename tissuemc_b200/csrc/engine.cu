// Host driver and C ABI of the B200 photon-walk engine (include/tissuemc_b200.h).
//
// Replaces TissueMC's src/cuda/engine.cu:322-358 (run_cuda) and :193-313 (run_with_tallies):
// the same validation and error texts, one persistent launch of walk_kernel, integer tallies
// decoded into the reference's result layout plus the 2-D arrays.

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/tissuemc_b200.h"
#include "walk_kernel.cuh"
#include "engine_host.hpp"
#include "engine_internal.hpp"

namespace tmc {

namespace {

constexpr int kMaxDevices = 64;

class Fail : public std::runtime_error {
  public:
    Fail(int code, const std::string &msg) : std::runtime_error(msg), code_(code) {}
    int code() const { return code_; }

  private:
    int code_;
};

#define TMC_CUDA(call)                                                                              \
    do {                                                                                            \
        const cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                      \
            throw Fail(TMC_CUDA_ERROR, std::string("CUDA error at ") + __FILE__ + ":" +             \
                                           std::to_string(__LINE__) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// Per-device state kept across calls: a stream, timing events, the tally buffer, the claim
// counter and a pinned staging buffer. Grown on demand, never shrunk.
struct DeviceCtx {
    bool ready = false;
    cudaDeviceProp prop{};
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    unsigned long long *d_tally = nullptr;
    size_t tally_cap = 0;  // words
    unsigned long long *d_counter = nullptr;
    uint64_t *h_stage = nullptr;
    size_t stage_cap = 0;  // words
};

DeviceCtx g_ctx[kMaxDevices];
std::mutex g_mu;

// The walk kernel for a launch: fast or exact math, with or without a shared core tile of A(r,z).
const void *walk_kernel_for(bool fast, bool core, bool profiles = true) {
    if (!profiles) return fast ? reinterpret_cast<const void *>(walk_kernel_totals<1>)
                               : reinterpret_cast<const void *>(walk_kernel_totals<0>);
    if (fast) return core ? reinterpret_cast<const void *>(walk_kernel<1, true>) : reinterpret_cast<const void *>(walk_kernel<1, false>);
    return core ? reinterpret_cast<const void *>(walk_kernel<0, true>) : reinterpret_cast<const void *>(walk_kernel<0, false>);
}

// Every instantiation may use the device's whole opt-in shared memory per block.
cudaError_t allow_walk_smem(const cudaDeviceProp &prop) {
    for (int f = 0; f < 2; ++f)
        for (int k = 0; k < 3; ++k) {
            const cudaError_t e = cudaFuncSetAttribute(walk_kernel_for(f != 0, k == 1, k != 2),
                                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                       static_cast<int>(prop.sharedMemPerBlockOptin));
            if (e != cudaSuccess) return e;
        }
    return cudaSuccess;
}

// Blocks per SM the registers of the walk kernel allow: the instantiation without a core tile when
// the options rule the core tile out (tile_tz = -1), else the one with it (the larger of the two).
int walk_blocks_per_sm(bool fast, int threads, bool core) {
    int bps = 0;
    const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, walk_kernel_for(fast, core), threads, 0);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return bps;
}


void set_status(tmc_status *st, int code, const std::string &msg) {
    if (!st) return;
    st->code = code;
    std::snprintf(st->message, sizeof st->message, "%s", msg.c_str());
}

DeviceCtx &device_ctx(int dev) {
    if (dev < 0 || dev >= kMaxDevices) throw Fail(TMC_BAD_CONFIG, "device ordinal out of range");
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
        cudaGetLastError();
        throw Fail(TMC_NO_DEVICE, "no usable CUDA device found");
    }
    if (dev >= n) throw Fail(TMC_NO_DEVICE, "no usable CUDA device found");
    TMC_CUDA(cudaSetDevice(dev));
    DeviceCtx &c = g_ctx[dev];
    if (!c.ready) {
        TMC_CUDA(cudaGetDeviceProperties(&c.prop, dev));
        TMC_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
        TMC_CUDA(cudaEventCreate(&c.ev0));
        TMC_CUDA(cudaEventCreate(&c.ev1));
        TMC_CUDA(cudaMalloc(&c.d_counter, 64));
        TMC_CUDA(allow_walk_smem(c.prop));
        c.ready = true;
    }
    return c;
}

// Blocks of `kern` that can be resident on the whole device at once with this dynamic shared memory
// (at least one wave's worth of one block per SM, so a launch always makes progress).
uint64_t resident_blocks(const void *kern, const cudaDeviceProp &prop, int threads, size_t smem) {
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, threads, smem) != cudaSuccess) {
        cudaGetLastError();
        occ = 1;
    }
    return static_cast<uint64_t>(prop.multiProcessorCount) * static_cast<uint64_t>(std::max(1, occ));
}

DeviceLimits limits_of(const cudaDeviceProp &p) {
    return DeviceLimits{p.multiProcessorCount, p.sharedMemPerMultiprocessor, p.sharedMemPerBlockOptin,
                        p.reservedSharedMemPerBlock};
}

void ensure_tally(DeviceCtx &c, size_t words) {
    if (words <= c.tally_cap) return;
    if (c.d_tally) TMC_CUDA(cudaFree(c.d_tally));
    c.d_tally = nullptr;
    c.tally_cap = 0;
    TMC_CUDA(cudaMalloc(&c.d_tally, words * 8));
    c.tally_cap = words;
}

void ensure_stage(DeviceCtx &c, size_t words) {
    if (words <= c.stage_cap) return;
    if (c.h_stage) TMC_CUDA(cudaFreeHost(c.h_stage));
    c.h_stage = nullptr;
    c.stage_cap = 0;
    TMC_CUDA(cudaMallocHost(&c.h_stage, words * 8));
    c.stage_cap = words;
}

}  // namespace

// ------------------------------------------------------------------------------ planning
// Shared-memory plan: the layer table, then (if they fit in a quarter of the budget) the per-batch
// totals, then the profile tallies. When the whole of A(r,z), R_d(r,a) and T_t(r,a) fits, all of it
// is privatised; otherwise R_d and T_t get the first rows (exits concentrate near the axis) and
// A(r,z) a core tile plus its clamped last row and column (the bins that collect every deposit
// beyond the grid, the hottest of a deep or wide stack). Everything else goes to global atomics.
Plan make_plan(const tmc_run_spec &spec, const tmc_options &opt, const DeviceLimits &lim,
               int regs_blocks_per_sm) {
    Plan p{};
    const RunShape sh = shape_of(spec, opt);
    p.threads = opt.threads_per_block > 0 ? opt.threads_per_block : 256;
    const int bps = opt.blocks_per_sm > 0 ? opt.blocks_per_sm : std::max(1, regs_blocks_per_sm);
    p.blocks_per_sm = bps;
    size_t budget = opt.smem_budget > 0
                        ? static_cast<size_t>(opt.smem_budget)
                        : std::min(lim.smem_block_optin, lim.smem_sm / static_cast<size_t>(bps) - lim.reserved);
    budget &= ~static_cast<size_t>(15);
    const size_t layer_bytes = ((static_cast<size_t>(sh.nl) * sizeof(LayerC) + 15) / 16) * 16;
    const size_t ring_bytes = 4 * kRingWords * static_cast<size_t>(p.threads);  // random words per lane
    budget = std::max(budget, layer_bytes + ring_bytes + 16);
    size_t rem = budget - layer_bytes - ring_bytes - 16;
    const size_t batch_bytes = static_cast<size_t>(sh.nb) * (4 + sh.nl) * 8;
    // The batch totals come first (up to half of what is left): every photon publishes into its
    // batch's words, and photon ids are claimed in order, so the lanes of the whole device are in one
    // or two batches at a time; in global memory those same-address atomics serialise in L2 (skin5,
    // 192 threads x 6 blocks per SM: 921 ms with the totals in global memory, 619 ms in shared).
    p.batch_smem = batch_bytes <= rem / 2 ? 1 : 0;
    if (p.batch_smem) rem -= batch_bytes;
    const size_t nr = sh.nr, nz = sh.nz, na = sh.na;
    if (opt.profiles) {
        const size_t full_a = nr * nz * 8, full_ra = nr * na * 8;
        if (full_a + 2 * full_ra <= rem) {
            p.tr_a = sh.nr;
            p.tz_a = sh.nz;
            p.tr_rd = p.tr_tt = sh.nr;
        } else {
            // rows of R_d(r,a) and T_t(r,a): an eighth of the budget each, or as the options say
            size_t rows = std::min(full_ra, rem / 8) / (na * 8);
            if (opt.tile_ra_rows == -1) rows = 0;
            if (opt.tile_ra_rows > 0) rows = std::min<size_t>({nr, static_cast<size_t>(opt.tile_ra_rows), rem / 2 / (na * 8)});
            // the rows never take the cross's room: its bins (the clamped last row and column of
            // A(r,z)) are the hottest of a deep or wide stack, and in global memory their
            // same-address atomics serialise in L2 (skin5 without the cross: 5.6 s, with it 0.62 s)
            const size_t cross = (nr + nz) * 8;
            const bool want_cross = opt.tile_cross != -1;
            if (want_cross && rem >= cross) rows = std::min(rows, (rem - cross) / (2 * na * 8));
            p.tr_rd = p.tr_tt = static_cast<int>(rows);
            rem -= 2 * rows * na * 8;
            if (want_cross && rem >= cross) {
                p.cross = 1;
                rem -= cross;
            }
            if (opt.tile_tz >= 0 && (p.cross || !want_cross)) {
                // the core tile: tz depth bins (about 2 sqrt(words), or as the options say) by as
                // many radial rows as fit; without the cross it may reach the last row and column
                const size_t core = rem / 8;
                const size_t zmax = p.cross ? nz - 1 : nz, rmax = p.cross ? nr - 1 : nr;
                size_t tz = opt.tile_tz > 0 ? static_cast<size_t>(opt.tile_tz)
                                            : static_cast<size_t>(2.0 * std::sqrt(static_cast<double>(core)));
                tz = std::min(tz, zmax);
                size_t tr = tz > 0 ? std::min(rmax, core / tz) : 0;
                if (tr == 0 || tz == 0) tr = tz = 0;
                p.tr_a = static_cast<int>(tr);
                p.tz_a = static_cast<int>(tz);
            }
        }
    }
    p.grid = lim.sms * bps;
    return p;
}

size_t plan_smem_bytes(const WalkParams &P) { return static_cast<size_t>(smem_layout(P).total) * 8; }

// Layer constants in float, computed in the same order as the reference evaluates them.
void fill_layers(const tmc_run_spec &spec, LayerC *out) {
    double zacc = 0.0;
    for (int i = 0; i < spec.num_layers; ++i) {
        const tmc_layer &s = spec.layers[i];
        const double nt = i == 0 ? spec.n_above : spec.layers[i - 1].n;
        const double nb = i + 1 == spec.num_layers ? spec.n_below : spec.layers[i + 1].n;
        LayerC &L = out[i];
        L = LayerC{};
        L.mua = static_cast<float>(s.mua);
        L.mus = static_cast<float>(s.mus);
        L.mut = L.mua + L.mus;
        L.inv_mut = 1.0f / L.mut;
        L.absorb = L.mua / L.mut;
        L.z0 = static_cast<float>(zacc);
        zacc += s.d;
        L.z1 = static_cast<float>(zacc);
        L.g = static_cast<float>(s.g);
        L.hg_a = 1.0f - L.g * L.g;
        L.hg_b = 1.0f - L.g;
        L.hg_c = 2.0f * L.g;
        L.hg_d = 1.0f + L.g * L.g;
        L.inv_2g = L.g != 0.0f ? 1.0f / (2.0f * L.g) : 0.0f;
        L.n = static_cast<float>(s.n);
        L.n_up = static_cast<float>(nt);
        L.n_dn = static_cast<float>(nb);
        L.cc_up = static_cast<float>(s.n > nt ? std::sqrt(1.0 - (nt * nt) / (s.n * s.n)) : 0.0);
        L.cc_dn = static_cast<float>(s.n > nb ? std::sqrt(1.0 - (nb * nb) / (s.n * s.n)) : 0.0);
        L.rat_up = L.n / L.n_up;
        L.rat_dn = L.n / L.n_dn;
        const float ru = (L.n_up - L.n) / (L.n_up + L.n);
        L.rn_up = ru * ru;
        const float rd = (L.n_dn - L.n) / (L.n_dn + L.n);
        L.rn_dn = rd * rd;
    }
}

// Launch weight 1 - R_sp in float, as the reference's launch() computes it (physics.hpp:50-66).
float launch_weight(const tmc_run_spec &spec) {
    const float n0 = static_cast<float>(spec.n_above), n1 = static_cast<float>(spec.layers[0].n);
    const float r = (n0 - n1) / (n0 + n1);
    return 1.0f - r * r;
}

// Fill WalkParams from a validated run.
WalkParams make_params(const tmc_run_spec &spec, const tmc_options &opt, const Plan &pl,
                       unsigned long long *d_tally, unsigned int *d_counter) {
    const RunShape sh = shape_of(spec, opt);
    WalkParams P{};
    P.photons = sh.photons;
    P.id_base = 0u;
    P.seed = opt.seed;
    P.plan_base = static_cast<uint32_t>(sh.photons / static_cast<uint64_t>(sh.nb));
    P.plan_extra = static_cast<uint32_t>(sh.photons % static_cast<uint64_t>(sh.nb));
    P.plan_bnd = P.plan_extra * (P.plan_base + 1u);
    P.threads = static_cast<uint32_t>(pl.threads);
    P.nb = sh.nb;
    P.nl = sh.nl;
    P.nz = sh.nz;
    P.nr = sh.nr;
    P.na = sh.na;
    const TallyOffsets off = tally_offsets(sh);
    P.counter = d_counter;
    P.g_batch = d_tally + off.batch;
    P.g_arz = d_tally + off.a_rz;
    P.g_rd = d_tally + off.rd_ra;
    P.g_tt = d_tally + off.tt_ra;
    P.launch_w = launch_weight(spec);
    P.dz = static_cast<float>(spec.dz);
    P.dr = static_cast<float>(spec.dr);
    P.da = static_cast<float>(0.5 * 3.14159265358979323846 / spec.na);
    P.inv_dz = 1.0f / P.dz;
    P.inv_dr = 1.0f / P.dr;
    P.inv_da = 1.0f / P.da;
    P.tr_a = pl.tr_a;
    P.tz_a = pl.tz_a;
    P.tr_rd = pl.tr_rd;
    P.tr_tt = pl.tr_tt;
    P.cross = pl.cross;
    P.batch_smem = pl.batch_smem;
    P.profiles = opt.profiles ? 1 : 0;
    P.step_cap = opt.step_cap ? opt.step_cap : kDefaultStepCap;
    // ids a warp claims at once: one per lane, so that when the ids run out no warp is left holding
    // a backlog of unstarted photons while others idle
    P.chunk = 32;
    uint32_t k0 = static_cast<uint32_t>(opt.seed), k1 = static_cast<uint32_t>(opt.seed >> 32);
    for (int r = 0; r < 10; ++r) {  // Philox4x32 key schedule (Weyl increments)
        P.round_keys[2 * r] = k0;
        P.round_keys[2 * r + 1] = k1;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    fill_layers(spec, P.layers);
    return P;
}

namespace {

// Launch the walk on `stream` into `d_tally` (zeroed here), claiming photon ids from `counter`
// (zeroed here; a word no other launch in flight uses). Records ev0/ev1 around it if given.
// With count > 0, only photons [first, first + count) of the run are walked (a shard: the same
// streams and batches as in the whole run, so the shards' tallies add up to the run's).
void launch_walk(const tmc_run_spec &spec, const tmc_options &opt, DeviceCtx &c,
                 unsigned long long *d_tally, unsigned long long *counter, cudaStream_t stream, cudaEvent_t e0,
                 cudaEvent_t e1, uint64_t first = 0, uint64_t count = 0) {
    const RunShape sh = shape_of(spec, opt);
    const size_t words = tally_offsets(sh).total;
    const int threads = opt.threads_per_block > 0 ? opt.threads_per_block : 256;
    const int regs_bps = walk_blocks_per_sm(opt.fast_math != 0, threads, opt.tile_tz != -1);
    const Plan pl = make_plan(spec, opt, limits_of(c.prop), regs_bps);
    WalkParams P = make_params(spec, opt, pl, d_tally, reinterpret_cast<unsigned int *>(counter));
    if (count) {
        P.photons = count;
        P.id_base = static_cast<uint32_t>(first);
    }
    const size_t smem = plan_smem_bytes(P);
    if (smem > c.prop.sharedMemPerBlockOptin)
        throw Fail(TMC_BAD_CONFIG, "the tally plan does not fit in shared memory");
    // never more lanes than photons (whole blocks only), and never more blocks than can be resident
    // at once with this plan's shared memory: the kernel is persistent, a second wave would idle
    const void *kern = walk_kernel_for(opt.fast_math != 0, pl.tr_a > 0 && pl.tz_a > 0, P.profiles != 0);
    const uint64_t max_blocks = (P.photons + pl.threads - 1) / pl.threads;
    const int grid = static_cast<int>(
        std::min<uint64_t>({static_cast<uint64_t>(pl.grid), max_blocks, resident_blocks(kern, c.prop, pl.threads, smem)}));
    if (e0) TMC_CUDA(cudaEventRecord(e0, stream));
    TMC_CUDA(cudaMemsetAsync(d_tally, 0, words * 8, stream));
    TMC_CUDA(cudaMemsetAsync(counter, 0, 8, stream));
    void *args[] = {&P};
    TMC_CUDA(cudaLaunchKernel(kern, dim3(grid), dim3(pl.threads), args, smem, stream));
    if (e1) TMC_CUDA(cudaEventRecord(e1, stream));
}

}  // namespace

double run_single_loop(const tmc_run_spec *specs, const tmc_options *opts, int n, std::vector<uint64_t> *raw,
                       std::vector<size_t> *offsets) {
    std::lock_guard<std::mutex> lock(g_mu);
    std::vector<size_t> off(static_cast<size_t>(n) + 1, 0);
    for (int c = 0; c < n; ++c) off[c + 1] = off[c] + tally_offsets(shape_of(specs[c], opts[c])).total;
    DeviceCtx &c = device_ctx(opts[0].device);
    ensure_tally(c, off[n]);
    TMC_CUDA(cudaEventRecord(c.ev0, c.stream));
    for (int i = 0; i < n; ++i)
        launch_walk(specs[i], opts[i], c, c.d_tally + off[i], c.d_counter, c.stream, nullptr, nullptr);
    TMC_CUDA(cudaEventRecord(c.ev1, c.stream));
    TMC_CUDA(cudaStreamSynchronize(c.stream));
    float ms = 0.f;
    TMC_CUDA(cudaEventElapsedTime(&ms, c.ev0, c.ev1));
    if (raw) {
        raw->resize(off[n]);
        TMC_CUDA(cudaMemcpy(raw->data(), c.d_tally, off[n] * 8, cudaMemcpyDeviceToHost));
    }
    if (offsets) *offsets = off;
    return static_cast<double>(ms) / 1000.0;
}
// ------------------------------------------------------------- allocation-free entry point
// Some callers cannot allocate device memory: a framework that owns every byte of device memory
// through its own pool and forbids libraries from calling cudaMalloc, or a plugin host that gives
// each plugin a fixed memory budget. tmc_b200_run_static serves them: the walk's scratch (its
// photon-claim counter and the fixed-point tally accumulators) lives in the file-scope array
// below, which the CUDA runtime places in every device's memory when the library's module is
// loaded there and keeps until exit.
namespace {

// Restores the calling thread's current device when the call returns (every exit path).
struct DeviceGuard {
    int saved = -1;
    DeviceGuard() {
        if (cudaGetDevice(&saved) != cudaSuccess) {
            cudaGetLastError();
            saved = -1;
        }
    }
    ~DeviceGuard() {
        if (saved >= 0) cudaSetDevice(saved);
    }
};

constexpr size_t kStaticHeadWords = 32;  // word 0: claim counter; the tallies start 256 B in
__device__ __align__(256) unsigned long long g_static_scratch[kStaticHeadWords + TMC_B200_STATIC_SCRATCH_WORDS];

struct StaticDevice {
    bool ready = false;
    cudaDeviceProp prop{};
    unsigned long long *scratch = nullptr;  // device address of g_static_scratch on this device
};
StaticDevice g_static_dev[kMaxDevices];

// Once per device, with that device current: the array's device address (its name in host code
// is only a host-side stand-in) and the kernels' shared-memory limit.
StaticDevice &static_device(int dev) {
    if (dev < 0 || dev >= kMaxDevices) throw Fail(TMC_BAD_CONFIG, "device ordinal out of range");
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0 || dev >= n) {
        cudaGetLastError();
        throw Fail(TMC_NO_DEVICE, "no usable CUDA device found");
    }
    TMC_CUDA(cudaSetDevice(dev));
    StaticDevice &d = g_static_dev[dev];
    if (!d.ready) {
        TMC_CUDA(cudaGetDeviceProperties(&d.prop, dev));
        void *addr = nullptr;
        TMC_CUDA(cudaGetSymbolAddress(&addr, g_static_scratch));
        d.scratch = static_cast<unsigned long long *>(addr);
        TMC_CUDA(allow_walk_smem(d.prop));
        d.ready = true;
    }
    return d;
}

}  // namespace

}  // namespace tmc

// ================================================================================== C ABI
using namespace tmc;

extern "C" {

int tmc_b200_available(void) {
    int n = 0;
    const bool ok = cudaGetDeviceCount(&n) == cudaSuccess && n > 0;
    if (!ok) cudaGetLastError();
    return ok ? 1 : 0;
}

int tmc_b200_abi_version(void) { return TMC_B200_ABI_VERSION; }

const char *tmc_b200_version(void) { return "tissuemc-b200 0.1.0 (sm_100a)"; }

int tmc_b200_run(const tmc_run_spec *spec, const tmc_options *opt, tmc_result *res, tmc_status *st) {
    set_status(st, TMC_OK, "");
    if (!spec || !opt || !res) {
        set_status(st, TMC_BAD_ARGUMENT, "NULL argument");
        return TMC_BAD_ARGUMENT;
    }
    const auto t0 = std::chrono::steady_clock::now();
    std::lock_guard<std::mutex> lock(g_mu);
    try {
        validate_run(*spec, *opt);  // throws Fail-compatible ConfigFailure
        const RunShape sh = shape_of(*spec, *opt);
        const size_t words = tally_offsets(sh).total;
        DeviceCtx &c = device_ctx(opt->device);
        ensure_tally(c, words);
        ensure_stage(c, words);
        launch_walk(*spec, *opt, c, c.d_tally, c.d_counter, c.stream, c.ev0, c.ev1);
        TMC_CUDA(cudaMemcpyAsync(c.h_stage, c.d_tally, words * 8, cudaMemcpyDeviceToHost, c.stream));
        TMC_CUDA(cudaStreamSynchronize(c.stream));
        float ms = 0.f;
        TMC_CUDA(cudaEventElapsedTime(&ms, c.ev0, c.ev1));
        decode_tallies(*spec, *opt, c.h_stage, *res);
        res->kernel_seconds = static_cast<double>(ms) / 1000.0;
        std::snprintf(res->device, sizeof res->device, "%.100s (sm_%d%d)", c.prop.name, c.prop.major,
                      c.prop.minor);
        res->wall_seconds =
            std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        return TMC_OK;
    } catch (const ConfigFailure &e) {
        set_status(st, TMC_BAD_CONFIG, e.what());
        return TMC_BAD_CONFIG;
    } catch (const Fail &e) {
        set_status(st, e.code(), e.what());
        return e.code();
    } catch (const std::exception &e) {
        set_status(st, TMC_CUDA_ERROR, e.what());
        return TMC_CUDA_ERROR;
    }
}

int tmc_b200_run_device_range(const tmc_run_spec *spec, const tmc_options *opt, uint64_t first_photon,
                              uint64_t count, uint64_t *d_tally, void *stream, tmc_status *st) {
    set_status(st, TMC_OK, "");
    if (!spec || !opt || !d_tally) {
        set_status(st, TMC_BAD_ARGUMENT, "NULL argument");
        return TMC_BAD_ARGUMENT;
    }
    std::lock_guard<std::mutex> lock(g_mu);
    try {
        validate_run(*spec, *opt);
        const uint64_t total = shape_of(*spec, *opt).photons;
        if (count == 0 || first_photon >= total || count > total - first_photon)
            throw ConfigFailure("photon range [" + std::to_string(first_photon) + ", " +
                                std::to_string(first_photon + count) + ") is empty or beyond the run's " +
                                std::to_string(total) + " photons");
        DeviceCtx &c = device_ctx(opt->device);
        unsigned long long *tally = reinterpret_cast<unsigned long long *>(d_tally);
        const size_t words = tally_offsets(shape_of(*spec, *opt)).total;
        launch_walk(*spec, *opt, c, tally, tally + words, static_cast<cudaStream_t>(stream), nullptr, nullptr,
                    first_photon, count);
        return TMC_OK;
    } catch (const ConfigFailure &e) {
        set_status(st, TMC_BAD_CONFIG, e.what());
        return TMC_BAD_CONFIG;
    } catch (const Fail &e) {
        set_status(st, e.code(), e.what());
        return e.code();
    } catch (const std::exception &e) {
        set_status(st, TMC_CUDA_ERROR, e.what());
        return TMC_CUDA_ERROR;
    }
}

int tmc_b200_run_device(const tmc_run_spec *spec, const tmc_options *opt, uint64_t *d_tally,
                        void *stream, tmc_status *st) {
    set_status(st, TMC_OK, "");
    if (!spec || !opt || !d_tally) {
        set_status(st, TMC_BAD_ARGUMENT, "NULL argument");
        return TMC_BAD_ARGUMENT;
    }
    std::lock_guard<std::mutex> lock(g_mu);
    try {
        validate_run(*spec, *opt);
        DeviceCtx &c = device_ctx(opt->device);
        unsigned long long *tally = reinterpret_cast<unsigned long long *>(d_tally);
        const size_t words = tally_offsets(shape_of(*spec, *opt)).total;
        launch_walk(*spec, *opt, c, tally, tally + words, static_cast<cudaStream_t>(stream), nullptr, nullptr);
        return TMC_OK;
    } catch (const ConfigFailure &e) {
        set_status(st, TMC_BAD_CONFIG, e.what());
        return TMC_BAD_CONFIG;
    } catch (const Fail &e) {
        set_status(st, e.code(), e.what());
        return e.code();
    } catch (const std::exception &e) {
        set_status(st, TMC_CUDA_ERROR, e.what());
        return TMC_CUDA_ERROR;
    }
}

int tmc_b200_run_static(const tmc_run_spec *spec, const tmc_options *opt, tmc_result *res, tmc_status *st) {
    set_status(st, TMC_OK, "");
    if (!spec || !opt || !res || !res->raw) {
        set_status(st, TMC_BAD_ARGUMENT, "NULL argument (tmc_b200_run_static needs result->raw as well)");
        return TMC_BAD_ARGUMENT;
    }
    const auto t0 = std::chrono::steady_clock::now();
    std::lock_guard<std::mutex> lock(g_mu);
    try {
        validate_run(*spec, *opt);
        const RunShape sh = shape_of(*spec, *opt);
        const size_t words = tally_offsets(sh).total;
        const DeviceGuard keep_device;
        if (words > TMC_B200_STATIC_SCRATCH_WORDS) {
            throw Fail(TMC_BAD_CONFIG,
                       "this run needs " + std::to_string(words) + " tally words but the static scratch of "
                       "tmc_b200_run_static holds " + std::to_string(TMC_B200_STATIC_SCRATCH_WORDS) +
                       " (fewer batches or bins, or use tmc_b200_run)");
        }
        StaticDevice &d = static_device(opt->device);
        unsigned long long *counter = d.scratch;
        unsigned long long *tally = d.scratch + kStaticHeadWords;
        const int threads = opt->threads_per_block > 0 ? opt->threads_per_block : 256;
        const int regs_bps = walk_blocks_per_sm(opt->fast_math != 0, threads, opt->tile_tz != -1);
        const Plan pl = make_plan(*spec, *opt, limits_of(d.prop), regs_bps);
        WalkParams P = make_params(*spec, *opt, pl, tally, reinterpret_cast<unsigned int *>(counter));
        const size_t smem = plan_smem_bytes(P);
        if (smem > d.prop.sharedMemPerBlockOptin)
            throw Fail(TMC_BAD_CONFIG, "the tally plan does not fit in shared memory");
        const void *kern = walk_kernel_for(opt->fast_math != 0, pl.tr_a > 0 && pl.tz_a > 0, P.profiles != 0);
        const uint64_t max_blocks = (sh.photons + pl.threads - 1) / pl.threads;
        const int grid = static_cast<int>(std::min<uint64_t>(
            {static_cast<uint64_t>(pl.grid), max_blocks, resident_blocks(kern, d.prop, pl.threads, smem)}));
        // the array keeps the previous call's contents: the counter and the tallies start at zero
        TMC_CUDA(cudaMemsetAsync(d.scratch, 0, (kStaticHeadWords + words) * 8, 0));
        const auto k0 = std::chrono::steady_clock::now();
        void *args[] = {&P};
        TMC_CUDA(cudaLaunchKernel(kern, dim3(grid), dim3(pl.threads), args, smem, 0));
        TMC_CUDA(cudaStreamSynchronize(0));
        const auto k1 = std::chrono::steady_clock::now();
        TMC_CUDA(cudaMemcpy(res->raw, tally, words * 8, cudaMemcpyDeviceToHost));
        uint64_t *raw = res->raw;
        res->raw = nullptr;  // decode into the other arrays without copying raw onto itself
        decode_tallies(*spec, *opt, raw, *res);
        res->raw = raw;
        res->kernel_seconds = std::chrono::duration<double>(k1 - k0).count();
        std::snprintf(res->device, sizeof res->device, "%.100s (sm_%d%d)", d.prop.name, d.prop.major,
                      d.prop.minor);
        res->wall_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        return TMC_OK;
    } catch (const ConfigFailure &e) {
        set_status(st, TMC_BAD_CONFIG, e.what());
        return TMC_BAD_CONFIG;
    } catch (const Fail &e) {
        set_status(st, e.code(), e.what());
        return e.code();
    } catch (const std::exception &e) {
        set_status(st, TMC_CUDA_ERROR, e.what());
        return TMC_CUDA_ERROR;
    }
}

int tmc_b200_autotune(const tmc_run_spec *spec, tmc_options *opt, uint64_t sample_photons, tmc_plan *plan_out,
                      double *default_seconds, double *best_seconds, tmc_status *st) {
    set_status(st, TMC_OK, "");
    if (!spec || !opt) {
        set_status(st, TMC_BAD_ARGUMENT, "NULL argument");
        return TMC_BAD_ARGUMENT;
    }
    std::lock_guard<std::mutex> lock(g_mu);
    try {
        validate_run(*spec, *opt);
        DeviceCtx &c = device_ctx(opt->device);
        // the sample: the run's first photons, with its seed and (at most as many) batches
        tmc_options base = *opt;
        const uint64_t total = shape_of(*spec, *opt).photons;
        base.photons = std::max<uint64_t>(1, std::min<uint64_t>(total, sample_photons ? sample_photons : total));
        base.batches = static_cast<int32_t>(std::min<uint64_t>(static_cast<uint64_t>(base.batches), base.photons));
        ensure_tally(c, tally_offsets(shape_of(*spec, base)).total);
        auto regs_blocks = [&](const tmc_options &o) {
            return walk_blocks_per_sm(o.fast_math != 0, o.threads_per_block > 0 ? o.threads_per_block : 256,
                                      o.tile_tz != -1);
        };
        auto time_of = [&](const tmc_options &o) -> double {
            const Plan pl = make_plan(*spec, o, limits_of(c.prop), regs_blocks(o));
            if (plan_smem_bytes(make_params(*spec, o, pl, nullptr, nullptr)) > c.prop.sharedMemPerBlockOptin)
                return 1e30;  // not a plan this device can run
            double best = 1e30;
            for (int rep = 0; rep < 3; ++rep) {  // a warm-up, then the best of two
                launch_walk(*spec, o, c, c.d_tally, c.d_counter, c.stream, c.ev0, c.ev1);
                TMC_CUDA(cudaStreamSynchronize(c.stream));
                float ms = 0.f;
                TMC_CUDA(cudaEventElapsedTime(&ms, c.ev0, c.ev1));
                if (rep) best = std::min(best, static_cast<double>(ms) / 1000.0);
            }
            return best;
        };
        const int regs_bps = regs_blocks(base);
        const Plan p0 = make_plan(*spec, base, limits_of(c.prop), regs_bps);
        tmc_options best = base;
        const double t_default = time_of(best);
        double t_best = t_default;
        auto try_opt = [&](const tmc_options &o) {
            const double t = time_of(o);
            if (t < t_best * 0.995) {  // keep a change only when it is clearly faster
                t_best = t;
                best = o;
            }
        };
        // coordinate descent: occupancy and block size first (they set the budget per block), then
        // the tile shapes within that budget
        for (int bps = std::max(1, regs_bps - 2); bps < regs_bps; ++bps) {
            tmc_options o = best;
            o.blocks_per_sm = bps;
            try_opt(o);
        }
        {
            tmc_options o = best;
            o.threads_per_block = 128;
            o.blocks_per_sm = 0;
            try_opt(o);
        }
        {
            tmc_options o = best;
            o.tile_cross = -1;
            try_opt(o);
        }
        const int tz0 = std::max(1, p0.tz_a);
        for (int tz : {-1, tz0 / 2, tz0 * 2, tz0 * 4, spec->nz}) {
            if (tz == 0) continue;
            tmc_options o = best;
            o.tile_tz = tz;
            try_opt(o);
        }
        const int rows0 = std::max(1, p0.tr_rd);
        for (int rows : {-1, rows0 / 2, rows0 * 2}) {
            if (rows == 0) continue;
            tmc_options o = best;
            o.tile_ra_rows = rows;
            try_opt(o);
        }
        // block sizes again, with the chosen tiles: without a core tile the kernel holds fewer
        // registers, and blocks of 6 or 7 warps fit more warps per SM than 8 (skin5: 36 warps of
        // 192-thread blocks, 0.75 % faster than 32 of 256 at full size)
        for (int threads : {192, 224, 128}) {
            if (threads == (best.threads_per_block > 0 ? best.threads_per_block : 256)) continue;
            tmc_options o = best;
            o.threads_per_block = threads;
            o.blocks_per_sm = 0;
            try_opt(o);
        }
        opt->threads_per_block = best.threads_per_block;
        opt->blocks_per_sm = best.blocks_per_sm;
        opt->tile_tz = best.tile_tz;
        opt->tile_ra_rows = best.tile_ra_rows;
        opt->tile_cross = best.tile_cross;
        if (plan_out) {
            const Plan p = make_plan(*spec, *opt, limits_of(c.prop), regs_blocks(*opt));
            const WalkParams P = make_params(*spec, *opt, p, nullptr, nullptr);
            *plan_out = tmc_plan{p.threads, p.blocks_per_sm, p.grid, p.tr_a, p.tz_a, p.cross, p.tr_rd, p.tr_tt,
                                 p.batch_smem, static_cast<int32_t>(plan_smem_bytes(P))};
        }
        if (default_seconds) *default_seconds = t_default;
        if (best_seconds) *best_seconds = t_best;
        return TMC_OK;
    } catch (const ConfigFailure &e) {
        set_status(st, TMC_BAD_CONFIG, e.what());
        return TMC_BAD_CONFIG;
    } catch (const Fail &e) {
        set_status(st, e.code(), e.what());
        return e.code();
    } catch (const std::exception &e) {
        set_status(st, TMC_CUDA_ERROR, e.what());
        return TMC_CUDA_ERROR;
    }
}

int tmc_b200_plan(const tmc_run_spec *spec, const tmc_options *opt, int32_t sms, int64_t smem_per_sm,
                  int64_t smem_per_block_optin, int64_t reserved_per_block, int32_t regs_blocks_per_sm,
                  tmc_plan *out, tmc_status *st) {
    set_status(st, TMC_OK, "");
    if (!spec || !opt || !out || sms < 1 || smem_per_sm < 1024 || smem_per_block_optin < 1024 ||
        reserved_per_block < 0) {
        set_status(st, TMC_BAD_ARGUMENT, "NULL argument or impossible device limits");
        return TMC_BAD_ARGUMENT;
    }
    try {
        validate_run(*spec, *opt);
        const DeviceLimits lim{sms, static_cast<size_t>(smem_per_sm), static_cast<size_t>(smem_per_block_optin),
                               static_cast<size_t>(reserved_per_block)};
        const Plan p = make_plan(*spec, *opt, lim, regs_blocks_per_sm);
        const WalkParams P = make_params(*spec, *opt, p, nullptr, nullptr);
        out->threads = p.threads;
        out->blocks_per_sm = p.blocks_per_sm;
        out->grid = p.grid;
        out->tr_a = p.tr_a;
        out->tz_a = p.tz_a;
        out->cross = p.cross;
        out->tr_rd = p.tr_rd;
        out->tr_tt = p.tr_tt;
        out->batch_smem = p.batch_smem;
        out->smem_bytes = static_cast<int32_t>(plan_smem_bytes(P));
        return TMC_OK;
    } catch (const ConfigFailure &e) {
        set_status(st, TMC_BAD_CONFIG, e.what());
        return TMC_BAD_CONFIG;
    }
}

}  // extern "C"
