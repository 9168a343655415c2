// Device side of the B200 photon walk: the per-lane state machine and one MCML step.
//
// Step semantics follow TissueMC's include/tissuemc/physics.hpp (launch :58-66, Fresnel :71-98,
// Henyey-Greenstein :101-113, spin :116-144, step size :148-158, boundary :162-178, hop :180-184,
// drop :187-193, crossing :198-246, roulette :250-259, step_once :263-277) and its Philox stream
// (include/tissuemc/philox.hpp:49-57, 91-122, 133-136), so photon i sees the same random words as
// on the CPU. The structure is this engine's own:
//
//  * a lane is one thread of a persistent, warp-synchronous loop; a lane whose photon ends claims
//    the next id from a per-warp pool, which the warp refills from a global counter in chunks;
//  * all photon state and the hot constants of the current layer live in registers; the random
//    words wait in a 16-word ring per lane in shared memory (walk_step.cuh, Ring), refilled with
//    one Philox block by every lane of the warp with room for it whenever any lane has fewer than
//    the four a step may draw; the layer table lives in shared memory and is read only when a
//    packet changes layer or meets a boundary;
//  * every tally is an unsigned 64-bit fixed-point integer (weight * 2^32, rounded), so sums are
//    exact and a run's output does not depend on scheduling; per-photon values (events, absorbed
//    weight in the current layer, the exit weight) accumulate in registers and are published once
//    per photon (or per layer change) into per-block shared-memory batch totals.
#pragma once

#include <cstdint>

namespace tmc {

constexpr int kMaxLayers = 16;
constexpr float kFixedScale = 4294967296.0f;  // 2^32
constexpr uint32_t kDefaultStepCap = 2000000000u;  // steps after which a live packet is an anomaly

// Constants of one layer, computed on the host in float arithmetic in the same order as the
// reference evaluates them (so e.g. hg_a is exactly float(1) - g * g). Laid out as six 16-byte
// groups: the first three are what a packet keeps in registers while it is in the layer (three
// 16-byte loads on entering it); the next two describe the boundary toward each side (one 16-byte
// load for the side a packet meets).
struct __align__(16) LayerC {
    float inv_mut, absorb, z0, z1;    // 1 / mu_t, mu_a / mu_t, top and bottom depth [cm]
    float g, hg_a, hg_b, hg_c;        // g, 1 - g*g, 1 - g, 2*g
    float hg_d, inv_2g, mut, mua;     // 1 + g*g, 1 / (2*g) (0 when g == 0), mu_a + mu_s, mu_a
    float n_up, rat_up, cc_up, rn_up; // toward the top: the neighbour's index (ambient at the end),
                                      // n / n_up, the critical cosine (0 if none), the
                                      // normal-incidence Fresnel reflectance
    float n_dn, rat_dn, cc_dn, rn_dn; // the same toward the bottom
    float n, mus, pad[2];             // this layer's index, mu_s
};
static_assert(sizeof(LayerC) == 24 * 4, "LayerC layout");

// Everything the walk kernel needs, passed by value (__grid_constant__).
struct WalkParams {
    uint64_t photons;      // photons of this launch: ids [id_base, id_base + photons), at most 2^31
    uint64_t seed;         // Philox key
    uint32_t plan_base;    // BatchPlan: photons per batch before the remainder
    uint32_t plan_extra;   // BatchPlan: the first `extra` batches hold one more
    uint32_t plan_bnd;     // BatchPlan: ids below extra * (base + 1) are in the larger batches
    uint32_t threads;      // block size (the random-word ring's stride)
    uint32_t id_base;      // first photon id (0 for a whole run; a shard of a run starts later)
    unsigned int *counter; // next unclaimed photon id (zeroed before launch)
    unsigned long long *g_batch;   // [nb * (4 + nl)] rd, tt, events, anomalies, absorbed[nl]
    unsigned long long *g_arz;     // [nr * nz]
    unsigned long long *g_rd;      // [nr * na]
    unsigned long long *g_tt;      // [nr * na]
    int nb, nl, nz, nr, na;
    float launch_w;        // 1 - specular reflectance, in float as the reference's launch()
    float dz, dr, da;      // bin widths (da = pi / (2 na))
    float inv_dz, inv_dr, inv_da;
    int tr_a, tz_a;        // shared tile of A(r,z): ir < tr_a and iz < tz_a
    int tr_rd, tr_tt;      // shared tiles of R_d(r,a) and T_t(r,a): ir < tr (all angles)
    int cross;             // 1: the clamped last row and column of A(r,z) are in shared memory too
    int batch_smem;        // 1: per-batch totals in shared memory
    int profiles;          // 0: skip A(r,z), R_d(r,a), T_t(r,a)
    uint32_t step_cap;     // a packet still alive after this many steps is ended as an anomaly
    int chunk;             // photon ids claimed per warp refill (>= 32)
    uint32_t round_keys[20];  // Philox key schedule of `seed` (k0, k1 of rounds 0..9), so that the
                              // rounds read their keys from the parameter bank instead of adding
    LayerC layers[kMaxLayers];
};

// ------------------------------------------------------------------------------------ Philox
__device__ __forceinline__ void philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t k0,
                                              uint32_t k1, uint32_t &o0, uint32_t &o1,
                                              uint32_t &o2, uint32_t &o3) {
    uint32_t c3 = 0u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = static_cast<uint64_t>(0xD2511F53u) * c0;
        const uint64_t p1 = static_cast<uint64_t>(0xCD9E8D57u) * c2;
        const uint32_t n0 = static_cast<uint32_t>(p1 >> 32) ^ c1 ^ k0;
        const uint32_t n2 = static_cast<uint32_t>(p0 >> 32) ^ c3 ^ k1;
        c0 = n0;
        c1 = static_cast<uint32_t>(p1);
        c2 = n2;
        c3 = static_cast<uint32_t>(p0);
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    o0 = c0;
    o1 = c1;
    o2 = c2;
    o3 = c3;
}

// The same rounds with the key schedule given (round r uses rk[2r], rk[2r + 1]).
__device__ __forceinline__ void philox4x32_10_rk(uint32_t c0, uint32_t c1, uint32_t c2, const uint32_t (&rk)[20],
                                                 uint32_t &o0, uint32_t &o1, uint32_t &o2, uint32_t &o3) {
    uint32_t c3 = 0u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = static_cast<uint64_t>(0xD2511F53u) * c0;
        const uint64_t p1 = static_cast<uint64_t>(0xCD9E8D57u) * c2;
        const uint32_t n0 = static_cast<uint32_t>(p1 >> 32) ^ c1 ^ rk[2 * r];
        const uint32_t n2 = static_cast<uint32_t>(p0 >> 32) ^ c3 ^ rk[2 * r + 1];
        c0 = n0;
        c1 = static_cast<uint32_t>(p1);
        c2 = n2;
        c3 = static_cast<uint32_t>(p0);
    }
    o0 = c0;
    o1 = c1;
    o2 = c2;
    o3 = c3;
}

// The key schedule of `key` (k0, k1 of rounds 0..9: k + r * (0x9E3779B9, 0xBB67AE85)) stored for
// one lane as five 16-byte words in shared memory, sched[q * stride] = rounds 2q and 2q + 1; a
// warp's load of word q reads 32 consecutive 16-byte words (no bank conflict).
__device__ __forceinline__ void key_schedule_store(uint4 *sched, int stride, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int q = 0; q < 5; ++q) {
        sched[q * stride] = make_uint4(k0, k1, k0 + 0x9E3779B9u, k1 + 0xBB67AE85u);
        k0 += 2u * 0x9E3779B9u;
        k1 += 2u * 0xBB67AE85u;
    }
}

// The same rounds with the key schedule read from shared memory (key_schedule_store): for lanes
// whose keys differ, where a schedule in the parameter bank cannot serve them all.
__device__ __forceinline__ void philox4x32_10_sched(uint32_t c0, uint32_t c1, uint32_t c2, const uint4 *sched,
                                                    int stride, uint32_t &o0, uint32_t &o1, uint32_t &o2,
                                                    uint32_t &o3) {
    uint32_t c3 = 0u;
#pragma unroll
    for (int q = 0; q < 5; ++q) {
        const uint4 k = sched[q * stride];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const uint64_t p0 = static_cast<uint64_t>(0xD2511F53u) * c0;
            const uint64_t p1 = static_cast<uint64_t>(0xCD9E8D57u) * c2;
            const uint32_t n0 = static_cast<uint32_t>(p1 >> 32) ^ c1 ^ (h ? k.z : k.x);
            const uint32_t n2 = static_cast<uint32_t>(p0 >> 32) ^ c3 ^ (h ? k.w : k.y);
            c0 = n0;
            c1 = static_cast<uint32_t>(p1);
            c2 = n2;
            c3 = static_cast<uint32_t>(p0);
        }
    }
    o0 = c0;
    o1 = c1;
    o2 = c2;
    o3 = c3;
}

// Uniform on (0,1) from one word, keeping 23 bits (philox.hpp:133-136).
// The value is ((x >> 9) + 1/2) * 2^-23, computed without an integer-to-float conversion: the 23
// kept bits become the mantissa of a float in [1, 2), 1 + m 2^-23, and subtracting 1 - 2^-24 gives
// (2m + 1) 2^-24 exactly (an odd integer below 2^24 times a power of two), bit for bit the
// reference's value.
__device__ __forceinline__ float unit_open(uint32_t x) {
#if TMC_UNIT_ADD
    // the same bits: (x >> 9) has no bit in common with the exponent pattern, so + equals |
    return __fsub_rn(__uint_as_float((x >> 9) + 0x3F800000u), 0x1.fffffep-1f);
#else
    return __fsub_rn(__uint_as_float((x >> 9) | 0x3F800000u), 0x1.fffffep-1f);
#endif
}

// ------------------------------------------------------------------------------------ math
// The walk is compiled in two variants: exact (MODE 0: IEEE division and square root, the
// accurate logf/sincosf, the reference's operation order) and fast (MODE 1). What "fast" replaces
// is the bit mask TMC_FAST_MASK, chosen so that the fast variant still meets the reference's
// identical-photon limits against the float32 CPU engine:
//   1: __logf for the step length          2: __sincosf for the azimuth
//   4: SFU reciprocal division and precomputed reciprocals (1/mu_t, mu_a/mu_t, 1/(2g), 10 for 1/0.1)
//   8: sqrt.approx and rsqrt (renormalisation, Fresnel, radius)
#ifndef TMC_FAST_MASK
#define TMC_FAST_MASK 15
#endif

template <int MODE> struct Math {
    static constexpr int mask = MODE ? TMC_FAST_MASK : 0;
    static constexpr bool log = (mask & 1) != 0;
    static constexpr bool sincos = (mask & 2) != 0;
    static constexpr bool div = (mask & 4) != 0;
    static constexpr bool sqrt = (mask & 8) != 0;
};

template <int MODE> __device__ __forceinline__ float m_div(float a, float b) {
    if constexpr (Math<MODE>::div) return __fdividef(a, b);
    else return a / b;
}
template <int MODE> __device__ __forceinline__ float m_sqrt(float x) {
    if constexpr (Math<MODE>::sqrt) {
        float r;
        asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
        return r;
    } else {
        return sqrtf(x);
    }
}
template <int MODE> __device__ __forceinline__ float m_rsqrt(float x) {
    if constexpr (Math<MODE>::sqrt) return rsqrtf(x);
    else return 1.0f / sqrtf(x);
}
template <int MODE> __device__ __forceinline__ float m_log(float x) {
    if constexpr (Math<MODE>::log) return __logf(x);
    else return logf(x);
}

// The step's floating-point arithmetic is written with its rounding pinned: every product, sum and
// fused multiply-add is an explicit round-to-nearest intrinsic, which the compiler may not contract
// or split. Two kernels that share the step (the single run and the sweep) therefore compute every
// photon identically whatever their register budgets, and the sweep's tallies stay bit for bit those
// of single runs.
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float ffma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
// The same operations on pairs, one paired instruction each (f32x2: two independent lanes, each
// rounded exactly as the scalar operation above), for the x/y halves of positions and directions.
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 fmul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 ffma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

// a^2 + b^2 + c^2 and a^2 + b^2
__device__ __forceinline__ float norm2(float a, float b, float c) { return ffma(a, a, ffma(b, b, fmul(c, c))); }
__device__ __forceinline__ float norm2(float a, float b) { return ffma(a, a, fmul(b, b)); }
__device__ __forceinline__ float norm2(float2 ab, float c) { return norm2(ab.x, ab.y, c); }
__device__ __forceinline__ float norm2(float2 ab) { return norm2(ab.x, ab.y); }

__device__ __forceinline__ unsigned long long to_fixed(float w) {
    return __float2ull_rn(fmul(w, kFixedScale));
}


}  // namespace tmc
