// The persistent photon-walk kernel of one run (see walk.cuh for the design and the reference
// citations; the step itself is walk_step.cuh).
#pragma once

#include "walk_step.cuh"
#include "work_queue.cuh"

namespace tmc {

// 1 (default): route a deposit with selects and one generic-address atomic, no divergent paths; 0:
// branch to the shared or the global atomic. On skin5 the branching form measured 2.1 % slower with
// a shared core tile and 30 % slower (811 against 624 ms for 1e8 photons) without one, where the
// lanes of a warp split between the shared last row and column and global memory at most steps.
#ifndef TMC_DEPOSIT_GENERIC
#define TMC_DEPOSIT_GENERIC 1
#endif
// Steps a lane takes per pass of the persistent loop (the relaunch ballot and the lane's live test
// once per pass; a lane whose packet ends early in a pass waits out the rest of it). Measured on
// skin5: 1 597.9 ms, 2 588.5 ms, 3 581.0 ms, 4 682.7 ms (64 registers, the loop body four steps
// long).
#ifndef TMC_STEPS_PER_ITER
#define TMC_STEPS_PER_ITER 3
#endif

// Shared-memory layout of one block, in 64-bit words (offsets computed identically on the host).
struct SmemLayout {
    int ring, batch, core_a, lastz_a, lastr_a, rd, tt, layers, total;  // word offsets / total words
};

__host__ __device__ inline SmemLayout smem_layout(const WalkParams &P) {
    SmemLayout s;
    int off = 0;
    // each lane's random words: a ring of kRingWords 32-bit words
    s.ring = off;
    off += static_cast<int>(kRingWords / 2) * static_cast<int>(P.threads);
    s.batch = off;
    off += P.batch_smem ? P.nb * (4 + P.nl) : 0;
    s.core_a = off;
    off += P.tr_a * P.tz_a;
    // The clamped last depth bin and last radius bin of A(r,z) collect every deposit beyond the
    // grid; for a deep or wide stack they are the hottest bins, so a tile that does not cover the
    // whole grid carries them too (a "cross": core + last column + last row).
    const bool cross = P.profiles && P.cross;
    s.lastz_a = off;
    off += cross ? P.nr : 0;
    s.lastr_a = off;
    off += cross ? P.nz : 0;
    s.rd = off;
    off += P.tr_rd * P.na;
    s.tt = off;
    off += P.tr_tt * P.na;
    off = (off + 1) & ~1;  // 16-byte alignment for the layer table
    s.layers = off;
    off += (P.nl * static_cast<int>(sizeof(LayerC)) + 7) / 8;
    s.total = off;
    return s;
}

// Where one run's walk keeps its layer table and tallies: a shared-memory layer table, per-batch
// totals and profile tiles privatised in shared memory (the rest in global memory).
// CORE: the plan has a shared core tile of A(r,z) (tr_a, tz_a > 0); without one the kernel is a
// separate instantiation that does not test for it.
// PROF: the run keeps the profile tallies (A(r,z), R_d(r,a), T_t(r,a)); a run of totals only is an
// instantiation of its own, so the step carries no test for it.
template <int FAST, bool CORE, bool PROF> struct PlainCtx {
    const WalkParams &P;
    Ring ring;  // refilled with the launch's precomputed Philox key schedule (P.round_keys)
    uint32_t step_cap;
    const LayerC *layers;
    unsigned long long *bt;
    int bstride;
    unsigned long long *s_core, *s_lastz, *s_lastr, *s_rd, *s_tt;
    bool cross;
    static constexpr bool kPublishAtRelaunch = true;  // measured 2.4 % faster than in the step

    __device__ __forceinline__ void refill(Lane &L) const { ring.refill(L, P.round_keys); }
    __device__ __forceinline__ uint32_t draw(Lane &L) const { return ring.draw(L); }
    __device__ __forceinline__ void skip(Lane &L) const { ring.skip(L); }
    __device__ __forceinline__ uint32_t peek(const Lane &L) const { return ring.peek(L); }
    __device__ __forceinline__ const LayerC &layer(const Lane &, int l) const { return layers[l]; }
    __device__ __forceinline__ int num_layers(const Lane &) const { return P.nl; }
    __device__ __forceinline__ void batch_add(const Lane &L, int slot, unsigned long long v) const {
        atomicAdd(&bt[L.batch * bstride + slot], v);
    }

    // Deposit into A(r,z) at bin (ir, iz): the shared core tile, the shared cross, or global.
    __device__ __forceinline__ void deposit(int ir, int iz, unsigned long long v) const {
#if TMC_DEPOSIT_GENERIC
        // one generic-address atomic on the selected word (no divergent paths)
        unsigned long long *p = &P.g_arz[static_cast<size_t>(ir) * P.nz + iz];
        if (cross && ir == P.nr - 1) p = &s_lastr[iz];
        if (cross && iz == P.nz - 1) p = &s_lastz[ir];
        if (CORE && ir < P.tr_a && iz < P.tz_a) p = &s_core[ir * P.tz_a + iz];
        atomicAdd(p, v);
        return;
#endif
        if (CORE && ir < P.tr_a && iz < P.tz_a) {
            atomicAdd(&s_core[ir * P.tz_a + iz], v);
        } else if (cross && iz == P.nz - 1) {
            atomicAdd(&s_lastz[ir], v);
        } else if (cross && ir == P.nr - 1) {
            atomicAdd(&s_lastr[iz], v);
        } else {
            atomicAdd(&P.g_arz[static_cast<size_t>(ir) * P.nz + iz], v);
        }
    }

    // Every deposit goes straight to its word (shared tile or global): a per-lane cache of the last
    // bin (merging consecutive deposits into one bin) measured 4 % slower on skin5, its branch
    // costing more than the atomics it saved.
    __device__ __forceinline__ void absorb(const Lane &L, unsigned long long v) const {
        if constexpr (!PROF) return;
        const float rr = radius<FAST>(L.xy);
        int ir, iz;
        bins_rz<FAST>(rr, L.z, P.dr, P.dz, P.inv_dr, P.inv_dz, P.nr, P.nz, ir, iz);
        deposit(ir, iz, v);
    }

    __device__ __forceinline__ void exit(const Lane &L, int kind, unsigned long long v) const {
        if constexpr (!PROF) return;
        const float rr = radius<FAST>(L.xy);
        const int ir = bin_of<FAST>(rr, P.dr, P.inv_dr, P.nr);
        const int ia = bin_of<FAST>(acosf(fminf(fabsf(L.uz), 1.0f)), P.da, P.inv_da, P.na);
        if (kind == 1) {
            if (ir < P.tr_rd) atomicAdd(&s_rd[ir * P.na + ia], v);
            else atomicAdd(&P.g_rd[ir * P.na + ia], v);
        } else {
            if (ir < P.tr_tt) atomicAdd(&s_tt[ir * P.na + ia], v);
            else atomicAdd(&P.g_tt[ir * P.na + ia], v);
        }
    }
};

// Minimum resident blocks per SM the compiler must allow for; 0 leaves the register budget to
// the compiler (which then uses 63 registers: four 256-thread blocks per SM).
#ifndef TMC_WALK_MIN_BLOCKS
#define TMC_WALK_MIN_BLOCKS 0
#endif
#if TMC_WALK_MIN_BLOCKS > 0
#define TMC_WALK_BOUNDS __launch_bounds__(256, TMC_WALK_MIN_BLOCKS)
#else
#define TMC_WALK_BOUNDS __launch_bounds__(256)
#endif

template <int FAST, bool CORE, bool PROF>
__device__ __forceinline__ void walk_body(const WalkParams &P) {
    extern __shared__ __align__(16) unsigned long long smem[];
    const SmemLayout S = smem_layout(P);
    for (int i = S.batch + threadIdx.x; i < S.layers; i += blockDim.x) smem[i] = 0ull;
    {
        const float *src = reinterpret_cast<const float *>(P.layers);
        float *dst = reinterpret_cast<float *>(smem + S.layers);
        for (int i = threadIdx.x; i < P.nl * static_cast<int>(sizeof(LayerC) / 4); i += blockDim.x) dst[i] = src[i];
    }
    __syncthreads();
    PlainCtx<FAST, CORE, PROF> C{P,
                     Ring{reinterpret_cast<uint32_t *>(smem + S.ring) + ring_lane_offset()},
                     P.step_cap,
                     reinterpret_cast<const LayerC *>(smem + S.layers),
                     P.batch_smem ? smem + S.batch : P.g_batch,
                     4 + P.nl,
                     smem + S.core_a,
                     smem + S.lastz_a,
                     smem + S.lastr_a,
                     smem + S.rd,
                     smem + S.tt,
                     P.profiles && P.cross};

    const unsigned lane = threadIdx.x & 31u;
    const unsigned lt_mask = (1u << lane) - 1u;
    const uint32_t n_photons = static_cast<uint32_t>(P.photons);  // at most 2^31 (validated)
    const uint32_t chunk = static_cast<uint32_t>(P.chunk);

    WarpPool pool;                           // warp-uniform photon-id pool
    unsigned ex_mask = 0u;                   // warp-uniform: lanes with no photon left to take
    bool alive = false;
    bool held = false;  // L holds a photon whose totals are not yet published
    Lane L;

    for (;;) {
        // ---- relaunch: lanes without a photon take the next ids from the warp's pool
        const unsigned need = ~__ballot_sync(0xffffffffu, alive) & ~ex_mask;
        if (need) {
            if (((need >> lane) & 1u) && held) {  // the lane's last photon ended: publish it
                finish_photon(L, C);
                held = false;
            }
            const uint32_t n = static_cast<uint32_t>(__popc(need));
            const uint32_t rank = static_cast<uint32_t>(__popc(need & lt_mask));
            uint32_t base = 0u;
            if (pool.must_claim(n)) {  // one lane claims the next chunk for the warp
                const int leader = __ffs(need) - 1;
                if (static_cast<int>(lane) == leader) base = atomicAdd(P.counter, chunk);
                base = __shfl_sync(0xffffffffu, base, leader);
            }
            const uint32_t my = pool.take(n, rank, base, chunk);
            const bool mine = (need >> lane) & 1u;
            ex_mask |= __ballot_sync(0xffffffffu, mine && my >= n_photons);
            if (mine && my < n_photons) {
                const uint32_t id = P.id_base + my;  // the run's photon id: its stream and its batch
                launch(L, C, id, batch_of(id, P.plan_base, P.plan_extra, P.plan_bnd), P.launch_w);
                alive = true;
                held = true;
            }
        }
        if (ex_mask == 0xffffffffu) break;  // exhausted lanes hold no photon: the warp is done
        if (!alive) continue;
        {
            bool ended = false;
#pragma unroll
            for (int k = 0; k < TMC_STEPS_PER_ITER; ++k)
                if (!ended) ended = walk_step<FAST>(L, C);
            if (ended) alive = false;
        }
    }

    // ---- publish the block's shared tallies into the global ones (integer adds: exact)
    __syncthreads();
    const int bstride = 4 + P.nl;
    if (P.batch_smem) {
        for (int i = threadIdx.x; i < P.nb * bstride; i += blockDim.x) {
            const unsigned long long v = smem[S.batch + i];
            if (v) atomicAdd(&P.g_batch[i], v);
        }
    }
    for (int i = threadIdx.x; i < (CORE ? P.tr_a * P.tz_a : 0); i += blockDim.x) {
        const unsigned long long v = C.s_core[i];
        if (v) atomicAdd(&P.g_arz[static_cast<size_t>(i / P.tz_a) * P.nz + (i % P.tz_a)], v);
    }
    if (C.cross) {
        for (int i = threadIdx.x; i < P.nr; i += blockDim.x) {
            const unsigned long long v = C.s_lastz[i];
            if (v) atomicAdd(&P.g_arz[static_cast<size_t>(i) * P.nz + (P.nz - 1)], v);
        }
        for (int i = threadIdx.x; i < P.nz; i += blockDim.x) {
            const unsigned long long v = C.s_lastr[i];
            if (v) atomicAdd(&P.g_arz[static_cast<size_t>(P.nr - 1) * P.nz + i], v);
        }
    }
    for (int i = threadIdx.x; i < P.tr_rd * P.na; i += blockDim.x) {
        const unsigned long long v = C.s_rd[i];
        if (v) atomicAdd(&P.g_rd[i], v);
    }
    for (int i = threadIdx.x; i < P.tr_tt * P.na; i += blockDim.x) {
        const unsigned long long v = C.s_tt[i];
        if (v) atomicAdd(&P.g_tt[i], v);
    }
}

// The walk of a run with profile tallies (CORE: with a shared core tile of A(r,z)).
template <int FAST, bool CORE>
__global__ void TMC_WALK_BOUNDS walk_kernel(const __grid_constant__ WalkParams P) {
    walk_body<FAST, CORE, true>(P);
}

// The walk of a run of totals only (no profile tallies).
template <int FAST>
__global__ void TMC_WALK_BOUNDS walk_kernel_totals(const __grid_constant__ WalkParams P) {
    walk_body<FAST, false, false>(P);
}

}  // namespace tmc
