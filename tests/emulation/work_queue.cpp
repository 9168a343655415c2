// Host emulation of how the persistent kernels hand out work (tissuemc_b200/csrc/work_queue.cuh),
// with warps and lanes emulated on the CPU in random interleavings. Built and run by
// tests/test_work_queue.py; exits non-zero with a message on the first broken property.
//
// Walk kernel (walk_kernel.cuh): each emulated warp runs the kernel's loop one iteration at a
// time, in a random order of warps — lanes without a photon take ids from the warp's pool, the
// pool claims chunks from a shared counter, a lane keeps its photon for a random number of steps.
// Properties: every id in [0, N) is launched exactly once and none beyond; each warp claims at
// most one chunk that starts at or past N; all lanes compute the same pool update; ids map to
// the BatchPlan batches with the right sizes.
//
// Sweep (sweep_kernel.cuh, sweep.cu): the item queue covers every photon of every configuration
// exactly once for ragged photon counts, item sizes and band counts; each band's order is a
// permutation of that band, taken before the next band; the strides are coprime with the counts.

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "../../tissuemc_b200/csrc/work_queue.cuh"

namespace {

using tmc::WarpPool;

int g_failures = 0;

#define EXPECT(cond, ...)                                  \
    do {                                                   \
        if (!(cond)) {                                     \
            std::fprintf(stderr, "FAILED %s: ", #cond);    \
            std::fprintf(stderr, __VA_ARGS__);             \
            std::fprintf(stderr, "\n");                    \
            ++g_failures;                                  \
            return;                                        \
        }                                                  \
    } while (0)

int popcount(uint32_t x) { return __builtin_popcount(x); }

struct Warp {
    WarpPool pool;
    uint32_t ex = 0u, alive = 0u;
    int steps[32] = {};
    int claims_past_end = 0;
    bool done = false;
};

void walk_case(uint32_t N, int W, uint32_t chunk, uint32_t nb, uint64_t seed) {
    std::mt19937_64 rng(seed);
    std::vector<uint8_t> launched(N, 0);
    uint64_t counter = 0;  // the launch's claim counter
    const uint32_t base = N / nb, extra = N % nb, bnd = extra * (base + 1u);
    std::vector<uint64_t> per_batch(nb, 0);
    std::vector<Warp> warps(static_cast<size_t>(W));
    int done = 0;
    uint64_t iterations = 0;
    while (done < W) {
        EXPECT(++iterations < 100000000ull, "N=%u W=%d: the emulation does not terminate", N, W);
        Warp &w = warps[rng() % static_cast<uint64_t>(W)];
        if (w.done) continue;
        const uint32_t need = ~w.alive & ~w.ex;
        if (need) {
            const uint32_t n = static_cast<uint32_t>(popcount(need));
            uint32_t claimed = 0u;
            if (w.pool.must_claim(n)) {  // the leader's atomicAdd
                EXPECT(counter + chunk < (1ull << 32), "N=%u: the 32-bit counter would wrap", N);
                claimed = static_cast<uint32_t>(counter);
                counter += chunk;
                if (claimed >= N) ++w.claims_past_end;
            }
            WarpPool after;
            bool first = true;
            for (uint32_t lane = 0; lane < 32; ++lane) {  // every lane runs take(), as in the kernel
                const uint32_t rank = static_cast<uint32_t>(popcount(need & ((1u << lane) - 1u)));
                WarpPool p = w.pool;
                const uint32_t id = p.take(n, rank, claimed, chunk);
                if (first) {
                    after = p;
                    first = false;
                }
                EXPECT(p.next == after.next && p.end == after.end, "lanes disagree on the pool update");
                EXPECT(p.next <= p.end, "pool [%u, %u) inverted", p.next, p.end);
                if (!((need >> lane) & 1u)) continue;
                if (id >= N) {
                    w.ex |= 1u << lane;
                    continue;
                }
                EXPECT(!launched[id], "N=%u: photon %u launched twice", N, id);
                launched[id] = 1;
                const int b = tmc::batch_of(id, base, extra, bnd);
                EXPECT(b >= 0 && static_cast<uint32_t>(b) < nb, "photon %u: batch %d of %u", id, b, nb);
                const uint64_t first_id = static_cast<uint64_t>(b) * base + (static_cast<uint32_t>(b) < extra ? b : extra);
                const uint64_t size = base + (static_cast<uint32_t>(b) < extra ? 1u : 0u);
                EXPECT(id >= first_id && id < first_id + size, "photon %u outside its batch %d", id, b);
                ++per_batch[static_cast<size_t>(b)];
                w.alive |= 1u << lane;
                w.steps[lane] = 1 + static_cast<int>(rng() % 60);
            }
            w.pool = after;
        }
        if (w.ex == 0xffffffffu) {
            EXPECT(w.alive == 0u, "a warp finished with live lanes");
            w.done = true;
            ++done;
            continue;
        }
        for (uint32_t lane = 0; lane < 32; ++lane)  // one step of every live lane
            if (((w.alive >> lane) & 1u) && --w.steps[lane] == 0) w.alive &= ~(1u << lane);
    }
    for (uint32_t id = 0; id < N; ++id) EXPECT(launched[id], "N=%u: photon %u never launched", N, id);
    for (const Warp &w : warps) EXPECT(w.claims_past_end <= 1, "a warp claimed %d chunks past the end", w.claims_past_end);
    EXPECT(counter % chunk == 0 && counter >= N, "counter %llu", static_cast<unsigned long long>(counter));
    for (uint32_t b = 0; b < nb; ++b)
        EXPECT(per_batch[b] == base + (b < extra ? 1u : 0u), "batch %u holds %llu photons", b,
               static_cast<unsigned long long>(per_batch[b]));
}

void sweep_case(const std::vector<uint32_t> &photons, uint32_t item, uint32_t bands) {
    const uint32_t n_cfg = static_cast<uint32_t>(photons.size());
    std::vector<uint32_t> prefix(n_cfg + 1u, 0u);
    uint64_t total = 0;
    for (uint32_t c = 0; c < n_cfg; ++c) {
        prefix[c] = static_cast<uint32_t>(total);
        total += (photons[c] + item - 1u) / item;
    }
    prefix[n_cfg] = static_cast<uint32_t>(total);
    const tmc::SweepOrder order = tmc::sweep_order(static_cast<uint32_t>(total), bands);
    std::vector<std::vector<uint8_t>> covered(n_cfg);
    for (uint32_t c = 0; c < n_cfg; ++c) covered[c].assign(photons[c], 0);
    for (uint32_t idx = 0; idx < total; ++idx) {
        const uint32_t j = order.item(idx);  // inside the band of idx: bands are taken in order
        EXPECT(j / order.band == idx / order.band, "item %u of band %u lands in band %u", idx, idx / order.band,
               j / order.band);
        uint32_t cfg = 0, first = 0, end = 0;
        tmc::sweep_item(idx, order, item, n_cfg, prefix.data(), [&](uint32_t c) { return photons[c]; }, cfg, first,
                        end);
        EXPECT(cfg < n_cfg && first < end && end <= photons[cfg] && end - first <= item,
               "item %u -> cfg %u [%u, %u)", idx, cfg, first, end);
        for (uint32_t p = first; p < end; ++p) {
            EXPECT(!covered[cfg][p], "cfg %u photon %u handed out twice", cfg, p);
            covered[cfg][p] = 1;
        }
    }
    for (uint32_t c = 0; c < n_cfg; ++c)
        for (uint32_t p = 0; p < photons[c]; ++p) EXPECT(covered[c][p], "cfg %u photon %u never handed out", c, p);
}

uint64_t gcd(uint64_t a, uint64_t b) {
    while (b) {
        const uint64_t t = a % b;
        a = b;
        b = t;
    }
    return a;
}

}  // namespace

int main() {
    // walk: tiny and ragged runs, one warp to thousands, chunks of 32 and more, batch plans
    const struct {
        uint32_t N;
        int W;
        uint32_t chunk, nb;
    } walks[] = {{1, 1, 32, 1},       {31, 1, 32, 1},     {32, 1, 32, 2},      {33, 1, 32, 3},
                 {33, 4, 32, 33},     {1000, 7, 32, 10},  {1000, 7, 64, 1000}, {4097, 100, 32, 100},
                 {100000, 64, 64, 10}, {50000, 4736, 32, 7}, {1u << 18, 592, 256, 100}};
    uint64_t seed = 1;
    for (const auto &c : walks)
        for (int rep = 0; rep < 3; ++rep) walk_case(c.N, c.W, c.chunk, c.nb, seed++);

    // sweep: single photons, item-size edges, ragged random counts, thousands of configurations,
    // one band to more bands than items
    for (uint32_t bands : {1u, 3u, 16u, 1000u}) {
        sweep_case({1}, 256, bands);
        sweep_case({255, 256, 257, 512, 1}, 256, bands);
        std::mt19937_64 rng(7 + bands);
        for (uint32_t item : {1u, 7u, 64u, 256u, 1024u}) {
            std::vector<uint32_t> ph(1 + rng() % 300);
            for (uint32_t &p : ph) p = 1 + static_cast<uint32_t>(rng() % 5000);
            sweep_case(ph, item, bands);
        }
        std::vector<uint32_t> many(4096);
        for (uint32_t &p : many) p = 1 + static_cast<uint32_t>(rng() % 3000);
        sweep_case(many, 256, bands);
    }

    // every band's order is a permutation of the band, for item counts and band counts around
    // the edges (a last band shorter than the others, bands of one item)
    for (uint32_t total = 1; total < 3000; ++total)
        for (uint32_t bands : {1u, 2u, 7u, 16u}) {
            const tmc::SweepOrder order = tmc::sweep_order(total, bands);
            std::vector<uint8_t> seen(total, 0);
            for (uint32_t idx = 0; idx < total; ++idx) {
                const uint32_t j = order.item(idx);
                if (j >= total || seen[j]) {
                    std::fprintf(stderr, "FAILED: %u items in %u bands: item %u taken twice or out of range\n",
                                 total, bands, j);
                    ++g_failures;
                    return 1;
                }
                seen[j] = 1;
            }
        }

    // the item order's stride is coprime with every item count (so the order is a permutation)
    for (uint64_t total = 0; total < 200000; ++total) {
        const uint32_t p = tmc::sweep_perm(total);
        if (total < 2) {
            if (p != 1u) {
                std::fprintf(stderr, "FAILED: stride %u for %llu items\n", p, static_cast<unsigned long long>(total));
                ++g_failures;
            }
        } else if (gcd(p, total) != 1 || p >= total) {
            std::fprintf(stderr, "FAILED: stride %u not coprime with %llu items\n", p,
                         static_cast<unsigned long long>(total));
            ++g_failures;
            break;
        }
    }
    if (g_failures) return 1;
    std::printf("work queue emulation: all properties hold\n");
    return 0;
}
