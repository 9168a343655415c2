// How the persistent kernels hand out work: the photon-id pool of a warp (walk_kernel.cuh), the
// batch of a photon id, and the item queue of the batched sweep and its order (sweep_kernel.cuh,
// sweep.cu).
//
// The code has no CUDA intrinsics, so it compiles for the host as well: the warp-level choices
// (who claims, which lane gets which id) are made by the callers with ballots and shuffles, and
// these functions only do the arithmetic on warp-uniform state. tests/emulation/work_queue.cpp
// runs them with emulated warps and lanes in random interleavings on the CPU — the reference's
// idea of testing kernel logic as host-compilable policies (tests/cpp/test_gpu_emulation.cpp).
#pragma once

#include <cstdint>

#if defined(__CUDACC__)
#define TMC_HD __host__ __device__ __forceinline__
#else
#define TMC_HD inline
#endif

namespace tmc {

// Batch of photon id `id` under TissueMC's BatchPlan (include/tissuemc/batching.hpp:11-29): nb
// batches of `base` photons, the first `extra` of them one larger; ids below bnd = extra *
// (base + 1) fall in the larger batches.
TMC_HD int batch_of(uint32_t id, uint32_t base, uint32_t extra, uint32_t bnd) {
    return static_cast<int>(id < bnd ? id / (base + 1u) : extra + (id - bnd) / base);
}

// The photon ids a warp has claimed from the launch's global counter and not handed out yet:
// [next, end). Warp-uniform: every lane holds the same copy and applies the same updates.
struct WarpPool {
    uint32_t next = 0u, end = 0u;

    // n lanes want a photon: must a new chunk be claimed first?
    TMC_HD bool must_claim(uint32_t n) const { return end - next < n; }

    // The id for the lane of rank `rank` (0 .. n - 1) among the n wanting ones; `base` is the
    // chunk of `chunk` ids (chunk >= 32) claimed when must_claim(n), ignored otherwise. Ids of the
    // old pool go first, then those of the new chunk. Call once per lane with the same n and base:
    // the pool advances identically everywhere.
    TMC_HD uint32_t take(uint32_t n, uint32_t rank, uint32_t base, uint32_t chunk) {
        const uint32_t avail = end - next;
        uint32_t id;
        if (avail >= n) {
            id = next + rank;
            next += n;
        } else {
            id = rank < avail ? next + rank : base + (rank - avail);
            next = base + (n - avail);
            end = base + chunk;
        }
        return id;
    }
};

// The order in which the sweep's items are taken: the item range is cut into bands of `band`
// items (the last one may be shorter), taken one band after the other; inside a band, item idx
// maps to start + (idx - start) * p mod size with p coprime with the band's size (perm, or
// perm_last for a shorter last band), which spreads the warps at work over many configurations.
// The host lays configurations out so that the first bands hold the longest photons: those start
// early, and the launch does not end waiting for one long photon that started last.
struct SweepOrder {
    uint32_t total, band, perm, perm_last;

    TMC_HD uint32_t item(uint32_t idx) const {
        const uint32_t start = idx / band * band;
        const uint32_t size = total - start < band ? total - start : band;
        const uint32_t p = size == band ? perm : perm_last;
        return start + static_cast<uint32_t>((static_cast<uint64_t>(idx - start) * p) % size);
    }
};

// Item `idx` of the sweep's queue (0 <= idx < order.total), taken as order.item(idx).
// Configuration c owns items prefix[c] .. prefix[c + 1] - 1, each of item_photons photons (its last
// one fewer when photons_of(c) is not a multiple). Gives the configuration, its first photon and
// one past its last.
template <class PhotonsOf>
TMC_HD void sweep_item(uint32_t idx, const SweepOrder &order, uint32_t item_photons, uint32_t n_cfg,
                       const uint32_t *prefix, PhotonsOf photons_of, uint32_t &cfg, uint32_t &first,
                       uint32_t &end) {
    const uint32_t j = order.item(idx);
    uint32_t lo = 0u, hi = n_cfg;  // the c with prefix[c] <= j < prefix[c + 1]
    while (hi - lo > 1u) {
        const uint32_t mid = (lo + hi) >> 1;
        if (prefix[mid] <= j) lo = mid;
        else hi = mid;
    }
    first = (j - prefix[lo]) * item_photons;
    const uint32_t left = photons_of(lo) - first;
    cfg = lo;
    end = first + (left < item_photons ? left : item_photons);
}

// A stride for a band of `total` items: the first of a few large odd multipliers whose residue is
// coprime with `total` (1, the plain order, when none is or total < 2).
inline uint32_t sweep_perm(uint64_t total) {
    constexpr uint32_t kCandidates[] = {2654435761u, 2246822519u, 3266489917u, 668265263u, 374761393u};
    if (total < 2) return 1u;
    for (uint32_t p : kCandidates) {
        uint64_t a = p % total, b = total;
        while (b) {
            const uint64_t t = a % b;
            a = b;
            b = t;
        }
        if (a == 1) return static_cast<uint32_t>(p % total);
    }
    return 1u;
}

// The order for `total` items (total >= 1) in at most `bands` bands.
inline SweepOrder sweep_order(uint32_t total, uint32_t bands) {
    const uint32_t nb = bands < 1u ? 1u : (bands < total ? bands : total);
    const uint32_t band = (total + nb - 1u) / nb;
    const uint32_t last = total - (total - 1u) / band * band;
    return SweepOrder{total, band, sweep_perm(band), sweep_perm(last)};
}

}  // namespace tmc
