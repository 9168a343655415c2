// The batched sweep: thousands of independent tissue configurations in one persistent launch.
//
// No reference code exists for this (it is an addition of this engine); each configuration's
// photons follow exactly the single-run walk (walk_step.cuh) with the Philox key of that
// configuration, so a configuration's tallies are bit for bit those of a single run with the
// same seed, photons, batches and grid.
//
// Work is a queue of items (configuration, first photon, count): configuration c's photons in
// chunks of item_photons, numbered through a prefix sum and taken band by band, in a strided
// permutation inside each band (work_queue.cuh, SweepOrder), so that the warps at work at any
// moment are spread over many configurations (their tallies then rarely meet on one L2 line). The
// host lays the configurations out longest photons first, so the bands run from the configurations
// whose photons take the most steps to those whose photons take the fewest. A warp takes items one
// at a time and hands their photons to its idle lanes; every lane carries the configuration of its
// own photon (its Philox key schedule in shared memory, written when the lane changes
// configuration; the layer table pointer; the tally base), so a warp moves on to the next item
// while some of its lanes still finish photons of the previous one, and no lane waits for an item
// to drain. Tallies of configuration c live at tally + c * stride in the single-run layout (batch
// totals, A(r,z), R_d(r,a), T_t(r,a)), accumulated with 64-bit integer atomics in global memory
// (L2).
//
// Optionally (tile_r x tile_z > 0) each warp privatises the first tile_r x tile_z bins of A(r,z) of
// one configuration, the one of the item it took last, in shared memory: deposits of its lanes'
// photons of that configuration into those bins are shared-memory atomics. When the warp takes an
// item of another configuration, its lanes first hand any pending run-cache value for the tile
// over, then the warp adds the tile's non-zero words into the configuration's global tallies and
// clears it (integer sums: the totals are the same whichever way they are summed).
#pragma once

#include "walk_step.cuh"
#include "work_queue.cuh"

namespace tmc {

// One configuration, as the kernel reads it.
struct SweepConfigC {
    uint32_t photons, plan_base, plan_extra, plan_bnd;  // photons and their BatchPlan
    uint32_t k0, k1;                                     // Philox key: this configuration's seed
    float launch_w;                                      // 1 - specular reflectance (float)
    int nl;                                              // layers
    int layer_base;                                      // index of layer 0 in the layer table
    int pad[3];
};
static_assert(sizeof(SweepConfigC) == 48, "SweepConfigC layout");

// Per-sweep header in device memory (written by the sweep's host-to-device copy, so that one
// captured graph serves sweeps of different sizes).
struct SweepHeader {
    uint32_t n_cfg;         // configurations
    uint32_t item_photons;  // photons per item (the last item of a configuration may hold fewer)
    SweepOrder order;       // order.total items (configuration c has ceil(photons_c / item_photons))
                            // and the order in which they are taken
};

struct SweepParams {
    const SweepHeader *hdr;
    const SweepConfigC *cfgs;
    const uint32_t *prefix;         // [n_cfg + 1] first item of each configuration
    const LayerC *layers;
    unsigned int *item_counter;     // next unclaimed item (zeroed before launch)
    unsigned long long *tally;      // [configs * stride]
    int stride;                     // 64-bit words per configuration
    int nb, lmax, nz, nr, na;       // batches, layer slots per batch row, grid
    float dz, dr, da, inv_dz, inv_dr, inv_da;
    int profiles;
    uint32_t step_cap;
    uint32_t threads;
    int tile_r, tile_z;             // per-warp shared tile of A(r,z) (0: none)
};

constexpr int kNoCacheKey = 0x7FFFFFFF;  // the run cache is empty (tally word indices stay below)

// 0 (default): every deposit goes straight to its word; 1: a per-lane run cache merges consecutive
// deposits into one A(r,z) bin (measured 5 % slower on the 4096-configuration sweep: its branch
// costs more than the atomics it saves)
#ifndef TMC_SWEEP_RUN_CACHE
#define TMC_SWEEP_RUN_CACHE 0
#endif

// Steps a lane takes per pass of the sweep's loop (the relaunch ballot and the live test once per
// pass). Measured on the 4096-configuration sweep: 1 1.303 s, 2 1.305 s (the kernel, held to 64
// registers, spills), 3 1.286 s.
#ifndef TMC_SWEEP_STEPS_PER_ITER
#define TMC_SWEEP_STEPS_PER_ITER 3
#endif

// 1: an ended packet's totals are published when its lane relaunches (as in the single-run kernel)
// instead of in the step; measured 0.9 % slower with one step per pass and 0.5 % faster with three
// (within the noise, and the kernel spills), so 0
#ifndef TMC_SWEEP_PUBLISH_AT_RELAUNCH
#define TMC_SWEEP_PUBLISH_AT_RELAUNCH 0
#endif

template <int FAST, bool TILE, bool PROF> struct SweepCtx {
    const SweepParams &P;
    Ring ring;
    uint32_t step_cap;
    int a_off, rd_off, tt_off, bstride;  // word offsets inside one configuration's tallies
    // the configuration of this lane's current photon, and its Philox key schedule (shared memory)
    uint32_t cfg;
    uint4 *sched;
    int nl;
    const LayerC *layers;
    int t;  // word offset of the configuration's tallies in P.tally (they hold < 2^31 words)
    // run cache: word index into P.tally of the last A(r,z) bin (or -1 - its index in the warp's
    // tile), and its pending value
    int cache_key;
    unsigned long long cache_val;
    // the warp's tile (warp-uniform): its words, and the configuration it holds (none: 0xFFFFFFFF)
    unsigned long long *tile;
    uint32_t tile_cfg;
    int tile_t;  // tally offset of tile_cfg

    // where an ended packet is published (TMC_SWEEP_PUBLISH_AT_RELAUNCH): in the step by default
    static constexpr bool kPublishAtRelaunch = TMC_SWEEP_PUBLISH_AT_RELAUNCH != 0;

    __device__ __forceinline__ void refill(Lane &L) const { ring.refill(L, sched, static_cast<int>(P.threads)); }
    __device__ __forceinline__ uint32_t draw(Lane &L) const { return ring.draw(L); }
    __device__ __forceinline__ void skip(Lane &L) const { ring.skip(L); }
    __device__ __forceinline__ uint32_t peek(const Lane &L) const { return ring.peek(L); }
    __device__ __forceinline__ const LayerC &layer(const Lane &, int l) const { return layers[l]; }
    __device__ __forceinline__ int num_layers(const Lane &) const { return nl; }
    __device__ __forceinline__ void batch_add(const Lane &L, int slot, unsigned long long v) const {
        atomicAdd(&P.tally[t + L.batch * bstride + slot], v);
    }
    __device__ __forceinline__ void deposit(int key, unsigned long long v) const {
        // negative keys name the warp's tile, which only the TILE instantiation has
        if (TILE && key < 0) atomicAdd(&tile[-1 - key], v);
        else atomicAdd(&P.tally[key], v);
    }
    __device__ __forceinline__ void absorb(const Lane &L, unsigned long long v) {
        if constexpr (!PROF) return;
        const float rr = radius<FAST>(L.xy);
        int ir, iz;
        bins_rz<FAST>(rr, L.z, P.dr, P.dz, P.inv_dr, P.inv_dz, P.nr, P.nz, ir, iz);
        int key = t + a_off + ir * P.nz + iz;
        if constexpr (TILE) {
            if (cfg == tile_cfg && ir < P.tile_r && iz < P.tile_z) key = -1 - (ir * P.tile_z + iz);
        }
#if !TMC_SWEEP_RUN_CACHE
        deposit(key, v);
        return;
#endif
        if (key == cache_key) {
            cache_val += v;
        } else {
            if (cache_key != kNoCacheKey) deposit(cache_key, cache_val);
            cache_key = key;
            cache_val = v;
        }
    }
    __device__ __forceinline__ void flush_cache() {
        if (cache_key != kNoCacheKey) deposit(cache_key, cache_val);
        cache_key = kNoCacheKey;
    }
    // Whole warp: hand the tile's sums to the global tallies of its configuration and clear it.
    __device__ __forceinline__ void flush_tile(unsigned lane) {
        if (cache_key < 0) {  // a pending run-cache value aimed at the tile
            atomicAdd(&tile[-1 - cache_key], cache_val);
            cache_key = kNoCacheKey;
        }
        __syncwarp();
        if (tile_cfg != 0xFFFFFFFFu) {
            for (int i = static_cast<int>(lane); i < P.tile_r * P.tile_z; i += 32) {
                const unsigned long long w = tile[i];
                if (w) {
                    atomicAdd(&P.tally[tile_t + a_off + (i / P.tile_z) * P.nz + i % P.tile_z], w);
                    tile[i] = 0ull;
                }
            }
        }
        __syncwarp();
    }
    __device__ __forceinline__ void exit(const Lane &L, int kind, unsigned long long v) const {
        if constexpr (!PROF) return;
        const float rr = radius<FAST>(L.xy);
        const int ir = bin_of<FAST>(rr, P.dr, P.inv_dr, P.nr);
        const int ia = P.na > 1 ? bin_of<FAST>(acosf(fminf(fabsf(L.uz), 1.0f)), P.da, P.inv_da, P.na) : 0;
        atomicAdd(&P.tally[t + (kind == 1 ? rd_off : tt_off) + ir * P.na + ia], v);
    }
};

// Minimum resident 256-thread blocks per SM the compiler must allow for (0: no bound). A bound of
// 4 caps the kernel at 64 registers (four blocks per SM instead of three). The step's arithmetic has
// its rounding pinned (walk.cuh), so the register budget cannot change any photon's path: the
// tallies stay bit-identical to the single-run kernel's.
#ifndef TMC_SWEEP_MIN_BLOCKS
#define TMC_SWEEP_MIN_BLOCKS 4
#endif
#if TMC_SWEEP_MIN_BLOCKS > 0
#define TMC_SWEEP_BOUNDS __launch_bounds__(256, TMC_SWEEP_MIN_BLOCKS)
#else
#define TMC_SWEEP_BOUNDS __launch_bounds__(256)
#endif

// TILE: the per-warp shared tile of A(r,z) is on (P.tile_r, P.tile_z > 0); the kernel without it
// is a separate instantiation, so that the tile's bookkeeping costs nothing when it is off.
template <int FAST, bool TILE, bool PROF>
__device__ __forceinline__ void sweep_body(const SweepParams &P) {
    extern __shared__ __align__(16) unsigned long long smem[];
    SweepCtx<FAST, TILE, PROF> C{P,
                     Ring{reinterpret_cast<uint32_t *>(smem) + ring_lane_offset()},
                     P.step_cap,
                     P.nb * (4 + P.lmax),
                     P.nb * (4 + P.lmax) + P.nr * P.nz,
                     P.nb * (4 + P.lmax) + P.nr * P.nz + P.nr * P.na,
                     4 + P.lmax,
                     0xFFFFFFFFu,
                     // after the rings (kRingWords words per lane): 5 x 16 bytes of key schedule per lane
                     reinterpret_cast<uint4 *>(reinterpret_cast<uint32_t *>(smem) + kRingWords * P.threads) +
                         threadIdx.x,
                     1,
                     P.layers,
                     0,
                     kNoCacheKey,
                     0ull,
                     // after the key schedules: one tile per warp
                     reinterpret_cast<unsigned long long *>(reinterpret_cast<uint32_t *>(smem) +
                                                            (kRingWords + 20) * P.threads) +
                         static_cast<size_t>(threadIdx.x >> 5) * P.tile_r * P.tile_z,
                     0xFFFFFFFFu,
                     0};
    const unsigned lane = threadIdx.x & 31u;
    if constexpr (TILE) {
        for (int i = static_cast<int>(lane); i < P.tile_r * P.tile_z; i += 32) C.tile[i] = 0ull;
        __syncwarp();
    }
    const unsigned lt_mask = (1u << lane) - 1u;
    const SweepHeader &H = *P.hdr;  // read where an item is taken (rare), not held in registers

    // warp-uniform: the item being handed out
    uint32_t it_cfg = 0u, it_next = 0u, it_end = 0u;
    bool items_done = false;
    unsigned ex_mask = 0u;  // warp-uniform: lanes with no photon left to take
    bool alive = false;
    bool held = false;  // L holds an ended photon whose totals are not yet published
    Lane L;

    for (;;) {
        unsigned need = ~__ballot_sync(0xffffffffu, alive) & ~ex_mask;
        if constexpr (decltype(C)::kPublishAtRelaunch) {
            if (((need >> lane) & 1u) && held) {  // the lane's last photon ended: publish it
                finish_photon(L, C);
                held = false;
            }
        }
        while (need) {  // warp-uniform: hand out photons, taking new items as they run out
            const uint32_t avail = it_end - it_next;
            if (avail == 0u) {
                if (!items_done) {
                    const int leader = __ffs(need) - 1;
                    uint32_t idx = 0u;
                    if (static_cast<int>(lane) == leader) idx = atomicAdd(P.item_counter, 1u);
                    idx = __shfl_sync(0xffffffffu, idx, leader);
                    if (idx < H.order.total) {
                        sweep_item(idx, H.order, H.item_photons, H.n_cfg, P.prefix,
                                   [&](uint32_t c) { return P.cfgs[c].photons; }, it_cfg, it_next, it_end);
                        if (TILE && it_cfg != C.tile_cfg) {  // the tile follows the warp's item
                            C.flush_tile(lane);
                            C.tile_cfg = it_cfg;
                            C.tile_t = static_cast<int>(it_cfg) * P.stride;
                        }
                        continue;
                    }
                    items_done = true;
                }
                ex_mask |= need;
                break;
            }
            const uint32_t n = static_cast<uint32_t>(__popc(need));
            const uint32_t take = n < avail ? n : avail;
            const uint32_t rank = static_cast<uint32_t>(__popc(need & lt_mask));
            const bool mine = ((need >> lane) & 1u) && rank < take;
            if (mine) {
                const SweepConfigC cf = P.cfgs[it_cfg];
                const uint32_t id = it_next + rank;
                if (it_cfg != C.cfg) {  // the lane's key schedule follows its configuration
                    C.cfg = it_cfg;
                    key_schedule_store(C.sched, static_cast<int>(P.threads), cf.k0, cf.k1);
                }
                C.nl = cf.nl;
                C.layers = P.layers + cf.layer_base;
                C.t = static_cast<int>(it_cfg) * P.stride;
                const int batch = batch_of(id, cf.plan_base, cf.plan_extra, cf.plan_bnd);
                launch(L, C, id, batch, cf.launch_w);
                alive = true;
                held = true;
            }
            need &= ~__ballot_sync(0xffffffffu, mine);
            it_next += take;
        }
        if (ex_mask == 0xffffffffu) break;  // exhausted lanes hold no photon: the warp is done
        if (!alive) continue;
        {
            bool ended = false;
#pragma unroll
            for (int k = 0; k < TMC_SWEEP_STEPS_PER_ITER; ++k)
                if (!ended) ended = walk_step<FAST>(L, C);
            if (ended) alive = false;
        }
    }
    C.flush_cache();
    if constexpr (TILE) C.flush_tile(lane);
}

// The sweep with profile tallies (TILE: with the per-warp shared tile of A(r,z)).
template <int FAST, bool TILE>
__global__ void TMC_SWEEP_BOUNDS sweep_kernel(const __grid_constant__ SweepParams P) {
    sweep_body<FAST, TILE, true>(P);
}

// The sweep of totals only (no profile tallies).
template <int FAST>
__global__ void TMC_SWEEP_BOUNDS sweep_kernel_totals(const __grid_constant__ SweepParams P) {
    sweep_body<FAST, false, false>(P);
}

// Per-configuration summaries from the integer tallies, in double: R_d(r) per photon (nr values,
// summed over exit angles), then total R_d, T_t and absorbed weight per photon. One warp per
// configuration; deterministic (integer sums, converted once).
__global__ void sweep_finalize_kernel(const SweepConfigC *cfgs, const unsigned long long *tally, int n_cfg,
                                      int stride, int nb, int lmax, int nz, int nr, int na, double *summary) {
    const int warp = static_cast<int>((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (warp >= n_cfg) return;
    const unsigned long long *t = tally + static_cast<size_t>(warp) * stride;
    const int bstride = 4 + lmax;
    const int rd_off = nb * bstride + nr * nz;
    const double k = 1.0 / (4294967296.0 * static_cast<double>(cfgs[warp].photons));
    double *out = summary + static_cast<size_t>(warp) * (nr + 3);
    for (int ir = lane; ir < nr; ir += 32) {
        unsigned long long s = 0ull;
        for (int ia = 0; ia < na; ++ia) s += t[rd_off + ir * na + ia];
        out[ir] = static_cast<double>(s) * k;
    }
    unsigned long long rd = 0ull, tt = 0ull, ab = 0ull;
    for (int b = lane; b < nb; b += 32) {
        rd += t[b * bstride + 0];
        tt += t[b * bstride + 1];
        for (int l = 0; l < lmax; ++l) ab += t[b * bstride + 4 + l];
    }
    for (int o = 16; o > 0; o >>= 1) {
        rd += __shfl_down_sync(0xffffffffu, rd, o);
        tt += __shfl_down_sync(0xffffffffu, tt, o);
        ab += __shfl_down_sync(0xffffffffu, ab, o);
    }
    if (lane == 0) {
        out[nr] = static_cast<double>(rd) * k;
        out[nr + 1] = static_cast<double>(tt) * k;
        out[nr + 2] = static_cast<double>(ab) * k;
    }
}

}  // namespace tmc
