// One MCML step of one lane, shared by the single-run kernel (walk_kernel.cuh) and the
// multi-configuration sweep kernel (sweep_kernel.cuh).
//
// Step semantics: TissueMC's include/tissuemc/physics.hpp — step size :148-158, boundary distance
// :162-178, hop :180-184, drop :187-193, Henyey-Greenstein :101-113, spin :116-144, Fresnel
// :71-98, crossing :198-246, roulette :250-259, step_once :263-277. A kernel supplies a context
// `Ctx` that says where the layer table and the tallies live:
//   ctx.refill(lane)          append the lane's next Philox block to its random-word ring
//   ctx.draw(lane)            next random word
//   ctx.layer(lane, l)        constants of layer l of the lane's tissue
//   ctx.num_layers(lane)
//   ctx.absorb(lane, v)       score an absorption of v (fixed point) at the lane's position
//   ctx.exit(lane, kind, v)   score an exit (1: reflectance, 2: transmittance) of v
//   ctx.batch_add(lane, i, v) add v to slot i of the lane's batch totals
//   ctx.step_cap              steps after which a packet is ended as an anomaly
//   Ctx::kPublishAtRelaunch   true: the kernel publishes an ended packet's totals (finish_photon)
//                             when the lane relaunches; false: the step does
#pragma once

#include "walk.cuh"

namespace tmc {

// Random words a lane keeps in its shared-memory ring (a power of two). With 16 (the default) the
// refill is warp-uniform: when any lane of the warp has fewer than the 4 words a step may draw,
// every lane with room for a block refills too, so the lanes of a warp refill together (0.75
// refills per step with all 32 lanes busy, against 1 per step with 24 of them when each lane
// refills on its own; measured 4.3 % faster on skin5). With 8 a lane refills alone. The words each
// photon consumes, and their order, are the same either way.
#ifndef TMC_RING_WORDS
#define TMC_RING_WORDS 16
#endif
constexpr uint32_t kRingWords = TMC_RING_WORDS;

// Where a packet keeps its layer's hot constants (Hot): 0 = in registers, loaded on entering a
// layer; 1 = read from the layer table (shared memory, three 16-byte loads) at every step, which
// frees twelve registers per lane for more resident warps.
#ifndef TMC_HOT_SMEM
#define TMC_HOT_SMEM 0
#endif
constexpr bool kHotInSmem = TMC_HOT_SMEM != 0;

static_assert(kRingWords == 8 || kRingWords == 16, "ring of 8 or 16 words");

constexpr float kCosZero = 1.0f - 1e-6f;  // physics.hpp:35 (float widening of MCML COSZERO)
constexpr float kCos90D = 1e-6f;          // physics.hpp:36
constexpr float kWeightMin = 1e-4f;       // physics.hpp:33 (MCML WEIGHT)
constexpr float kChance = 0.1f;           // physics.hpp:34 (MCML CHANCE)
constexpr float kTwoPi = 2.0f * 3.14159265358979323846f;  // evaluated as the reference does

// Register copy of the current layer's constants used on every step.
struct Hot {
    float mua, mut, inv_mut, absorb, z0, z1, g, hg_a, hg_b, hg_c, hg_d, inv_2g;
};

__device__ __forceinline__ void load_hot(Hot &h, const LayerC &L) {
    const float4 *q = reinterpret_cast<const float4 *>(&L);  // three 16-byte loads
    const float4 a = q[0], b = q[1], c = q[2];
    h.inv_mut = a.x;
    h.absorb = a.y;
    h.z0 = a.z;
    h.z1 = a.w;
    h.g = b.x;
    h.hg_a = b.y;
    h.hg_b = b.z;
    h.hg_c = b.w;
    h.hg_d = c.x;
    h.inv_2g = c.y;
    h.mut = c.z;
    h.mua = c.w;
}

// The boundary of layer L toward the top (up) or the bottom: the neighbour's index, the index
// ratio, the critical cosine and the normal-incidence reflectance, in one 16-byte load.
__device__ __forceinline__ float4 boundary_side(const LayerC &L, bool up) {
    return reinterpret_cast<const float4 *>(&L)[up ? 3 : 4];
}

// Fresnel reflectance for unpolarised light from index n1 into n2 at cos(incidence) ca1
// (physics.hpp:71-98); rn is the precomputed normal-incidence value and rat = n1 / n2.
template <int FAST>
__device__ __forceinline__ float fresnel(float n1, float n2, float ca1, float rn, float rat,
                                         float &ca2) {
    if (n1 == n2) {
        ca2 = ca1;
        return 0.0f;
    }
    if (ca1 > kCosZero) {
        ca2 = ca1;
        return rn;
    }
    if (ca1 < kCos90D) {
        ca2 = 0.0f;
        return 1.0f;
    }
    const float sa1 = m_sqrt<FAST>(ffma(-ca1, ca1, 1.0f));
    float sa2;
    if constexpr (Math<FAST>::div) sa2 = fmul(sa1, rat);
    else sa2 = fmul(n1, sa1) / n2;
    if (sa2 >= 1.0f) {
        ca2 = 0.0f;
        return 1.0f;
    }
    ca2 = m_sqrt<FAST>(ffma(-sa2, sa2, 1.0f));
    const float cc = fmul(ca1, ca2), ss = fmul(sa1, sa2), sc = fmul(sa1, ca2), cs = fmul(ca1, sa2);
    const float cap = fsub(cc, ss), cam = fadd(cc, ss), sap = fadd(sc, cs), sam = fsub(sc, cs);
    return m_div<FAST>(fmul(fmul(fmul(0.5f, sam), sam), norm2(cam, cap)), fmul(fmul(sap, sap), fmul(cam, cam)));
}

// Clamped bin index (src/cpu/engine.cpp:59-66 semantics, branch-free): x <= 0 or NaN -> 0,
// x / width >= n -> n - 1, else floor(x / width).
// The clamp is the conversion's own: a float-to-unsigned conversion that truncates turns negative
// values and NaN into 0 and saturates large ones, so min(u, n - 1) is the clamped bin.
__device__ __forceinline__ int clamp_bin(float i, int n) {
    return static_cast<int>(umin(__float2uint_rz(i), static_cast<unsigned>(n - 1)));
}
template <int FAST> __device__ __forceinline__ int bin_of(float x, float width, float inv_width, int n) {
    float i;
    if constexpr (Math<FAST>::div) i = fmul(x, inv_width);
    else i = x / width;
    return clamp_bin(i, n);
}
// The radius and depth bins of one deposit (r, z) together: in fast math the two products are one
// paired instruction.
template <int FAST>
__device__ __forceinline__ void bins_rz(float r, float z, float dr, float dz, float inv_dr, float inv_dz, int nr, int nz,
                                        int &ir, int &iz) {
    if constexpr (Math<FAST>::div) {
        const float2 i = fmul2(f2(r, z), f2(inv_dr, inv_dz));
        ir = clamp_bin(i.x, nr);
        iz = clamp_bin(i.y, nz);
    } else {
        ir = bin_of<FAST>(r, dr, inv_dr, nr);
        iz = bin_of<FAST>(z, dz, inv_dz, nz);
    }
}

// Free path -ln(u) / mu_t of an interaction step (physics.hpp:148-158).
template <int FAST> __device__ __forceinline__ float step_length(const Hot &h, float u) {
    if constexpr (Math<FAST>::log) {
        // the SFU logarithm's absolute error can flip the sign of log(u) for the two largest u of
        // the 23-bit grid; a step is never negative
        return fmul(fmaxf(-m_log<FAST>(u), 0.0f), h.inv_mut);
    } else if constexpr (Math<FAST>::div) {
        return fmul(-m_log<FAST>(u), h.inv_mut);
    } else {
        return -m_log<FAST>(u) / h.mut;
    }
}

// Henyey-Greenstein cosine of the scattering angle from one uniform draw (physics.hpp:101-113).
template <int FAST> __device__ __forceinline__ float hg_cos(const Hot &h, float xi) {
    const float t = m_div<FAST>(h.hg_a, ffma(h.hg_c, xi, h.hg_b));
    float ct;
    if constexpr (Math<FAST>::div) ct = fmul(ffma(-t, t, h.hg_d), h.inv_2g);
    else ct = ffma(-t, t, h.hg_d) / h.hg_c;
    // an isotropic layer selects 2 xi - 1 (the formula above is 0 / 0 there, clamped, then
    // discarded): a select instead of a branch, measured 1.0 % faster on skin5
    return h.g == 0.0f ? ffma(2.0f, xi, -1.0f) : fminf(fmaxf(ct, -1.0f), 1.0f);
}

// Turn the direction (u.x, u.y, uz) by the polar cosine ct and the azimuth 2 pi u, then renormalise
// it (physics.hpp:116-144). The x and y halves go through paired instructions, each half rounded as
// the scalar form would round it.
template <int FAST>
__device__ __forceinline__ void rotate(float2 &uxy, float &uz, float ct, float u) {
    float st = ffma(-ct, ct, 1.0f);
    st = st > 0.0f ? m_sqrt<FAST>(st) : 0.0f;
    float sp, cp;
    if constexpr (Math<FAST>::sincos) {
        // psi - pi lies in (-pi, pi), where the SFU sine and cosine are accurate
        __sincosf(fmul(kTwoPi, fsub(u, 0.5f)), &sp, &cp);
        sp = -sp;
        cp = -cp;
    } else {
        sincosf(fmul(kTwoPi, u), &sp, &cp);
    }
    if (fabsf(uz) > kCosZero) {
        uxy = fmul2(f2(st), f2(cp, sp));
        uz = uz >= 0.0f ? ct : -ct;
    } else {
        const float2 o = uxy;
        const float oz = uz;
        const float q = ffma(-oz, oz, 1.0f);  // 1 - uz^2
        // (ix, iy) = (ox oz cp - oy sp, oy oz cp + ox sp)
        const float2 ixy = ffma2(fmul2(o, f2(oz)), f2(cp), fmul2(f2(-o.y, o.x), f2(sp)));
        const float2 oct = fmul2(o, f2(ct));
        if constexpr (Math<FAST>::sqrt) {
            const float it = rsqrtf(q);
            uxy = ffma2(fmul2(f2(st), ixy), f2(it), oct);
            uz = ffma(fmul(fmul(-st, cp), q), it, fmul(oz, ct));
        } else {
            const float tmp = sqrtf(q);
            uxy = f2(fadd(fmul(st, ixy.x) / tmp, oct.x), fadd(fmul(st, ixy.y) / tmp, oct.y));
            uz = ffma(fmul(-st, cp), tmp, fmul(oz, ct));
        }
    }
    const float inv = m_rsqrt<FAST>(norm2(uxy, uz));
    uxy = fmul2(uxy, f2(inv));
    uz = fmul(uz, inv);
}

// Radial distance of the packet from the source axis (the r of A(r,z), R_d(r,a), T_t(r,a)).
template <int FAST> __device__ __forceinline__ float radius(float2 xy) { return m_sqrt<FAST>(norm2(xy)); }

// All state of one lane's current photon (registers).
struct Lane {
    float2 xy;   // position across the layers (x, y) [cm]
    float2 uxy;  // direction cosines (ux, uy)
    float z, uz, w, sleft;
    int layer, batch;
    uint32_t id, blk, rp, wp;  // photon id, Philox block, ring read/write positions
    uint32_t events, anomalies, steps;
    unsigned long long run_abs;  // fixed-point weight absorbed in the current layer
    Hot h;
};

// Launch a packet at the origin, straight down, in layer 0 (physics.hpp:58-66).
template <class Ctx>
__device__ __forceinline__ void launch(Lane &L, Ctx &C, uint32_t id, int batch, float launch_w) {
    L.id = id;
    L.blk = 0u;
    L.rp = L.wp = 0u;
    L.xy = f2(0.f);
    L.z = 0.f;
    L.uxy = f2(0.f);
    L.uz = 1.f;
    L.w = launch_w;
    L.sleft = 0.f;
    L.layer = 0;
    if constexpr (!kHotInSmem) load_hot(L.h, C.layer(L, 0));
    L.batch = batch;
    L.events = L.anomalies = L.steps = 0u;
    L.run_abs = 0ull;
}

// Publish an ended packet's per-photon totals (events, anomalies, the weight absorbed in its last
// layer) into its batch.
template <class Ctx> __device__ __forceinline__ void finish_photon(const Lane &L, Ctx &C) {
    C.batch_add(L, 2, static_cast<unsigned long long>(L.events));
    if (L.anomalies) C.batch_add(L, 3, static_cast<unsigned long long>(L.anomalies));
    if (L.run_abs) C.batch_add(L, 4 + L.layer, L.run_abs);
}

// The first part of a step: refill the random words, the free path (or what is left of it), the
// distance to the layer's boundary, and the hop. Returns true when the hop ends on the boundary.
// The layer constants of the packet's current layer (registers, or the layer table: kHotInSmem).
template <class Ctx> __device__ __forceinline__ Hot hot_of(const Lane &L, Ctx &C) {
    if constexpr (kHotInSmem) {
        Hot h;
        load_hot(h, C.layer(L, L.layer));
        return h;
    } else {
        return L.h;
    }
}

template <int FAST, class Ctx> __device__ __forceinline__ bool step_move(Lane &L, Ctx &C, const Hot &h) {
    if constexpr (kRingWords == 8) {
        if (L.wp - L.rp < 4u) C.refill(L);  // a step draws at most 4 words
    } else {
        // warp-uniform: the lanes stepping together refill together when any of them is short
        if (__any_sync(__activemask(), L.wp - L.rp < 4u) && L.wp - L.rp <= kRingWords - 4u) C.refill(L);
    }
    ++L.steps;
    float s;
    {
        // both candidates, then a select: a fresh free path (which consumes the next word) or the
        // rest of the one a boundary cut short (which consumes none). The word is read either way
        // (the ring always holds it) and passed over only when used. Half of a warp's steps hold a
        // lane that has just left a boundary, so a branch here diverged; the select measured 5.4 %
        // faster on skin5.
        const bool fresh = L.sleft == 0.0f;
        const float s_fresh = step_length<FAST>(h, unit_open(C.peek(L)));
        float s_rest;
        if constexpr (Math<FAST>::div) s_rest = fmul(L.sleft, h.inv_mut);
        else s_rest = L.sleft / h.mut;
        s = fresh ? s_fresh : s_rest;
        L.rp += fresh ? 1u : 0u;
        L.sleft = 0.0f;
    }
    // the distance to the boundary the packet heads for, and a select instead of a branch (measured
    // 1.2 % faster on skin5): with uz = 0 the quotient is infinite or NaN and the test discards it
    const float db = m_div<FAST>(fsub(L.uz > 0.0f ? h.z1 : h.z0, L.z), L.uz);
    const bool hit = L.uz != 0.0f && s > db;
    L.sleft = hit ? fmul(fsub(s, db), h.mut) : 0.0f;
    s = hit ? db : s;
    L.xy = ffma2(f2(s), L.uxy, L.xy);
    L.z = ffma(s, L.uz, L.z);
    return hit;
}

// At the boundary: reflect, or transmit into the next layer or out (physics.hpp:198-246). Sets
// exit_kind (1: reflectance, top; 2: transmittance, bottom) and died when the packet leaves.
template <int FAST, class Ctx>
__device__ __forceinline__ void step_boundary(Lane &L, Ctx &C, int &exit_kind, bool &died) {
    const LayerC &Lc = C.layer(L, L.layer);
    const bool up = L.uz < 0.0f;
    const float ca1 = up ? -L.uz : L.uz;
    const float4 side = boundary_side(Lc, up);  // n_t, n / n_t, critical cosine, normal-incidence R
    const float nt = side.x, rat = side.y;
    float uz1 = 0.0f;
    bool through;
    if (nt == Lc.n) {
        // matched indices: R = 0, so the Fresnel word (in (0, 1), always above R) is drawn and not
        // needed, and the direction goes through unchanged (rat = 1, cos_t = cos_i); measured 2.8 %
        // faster on skin5, whose inner boundaries are all matched
        C.skip(L);
        through = true;
        uz1 = ca1;
    } else {
        const float r = (ca1 <= side.z) ? 1.0f : fresnel<FAST>(Lc.n, nt, ca1, side.w, rat, uz1);
        through = unit_open(C.draw(L)) > r;
    }
    if (through) {
        L.uxy = fmul2(L.uxy, f2(rat));
        L.uz = up ? -uz1 : uz1;
        if (up ? L.layer == 0 : L.layer == C.num_layers(L) - 1) {
            exit_kind = up ? 1 : 2;
            died = true;
        } else {
            C.batch_add(L, 4 + L.layer, L.run_abs);  // adds 0 when nothing was absorbed: no branch
            L.run_abs = 0ull;
            L.layer += up ? -1 : 1;
            if constexpr (!kHotInSmem) load_hot(L.h, C.layer(L, L.layer));
        }
    } else {
        L.uz = -L.uz;
    }
}

// An interaction: drop (physics.hpp:187-193), score the absorption, spin (physics.hpp:101-144).
template <int FAST, class Ctx> __device__ __forceinline__ void step_interaction(Lane &L, Ctx &C, const Hot &h) {
    float dwa;
    if constexpr (Math<FAST>::div) dwa = fmul(L.w, h.absorb);
    else dwa = fmul(L.w, h.mua) / h.mut;
    L.w = fsub(L.w, dwa);
    ++L.events;
    {
        // a NaN weight turns the norm's deviation into NaN (0 * NaN), which fails the comparison
        const float n2 = norm2(L.uxy, L.uz);
        if (!(fabsf(ffma(dwa, 0.0f, fsub(n2, 1.0f))) <= 1e-5f)) ++L.anomalies;
    }
    const unsigned long long v = to_fixed(dwa);
    L.run_abs += v;
    C.absorb(L, v);
    const float ct = hg_cos<FAST>(h, unit_open(C.draw(L)));
    rotate<FAST>(L.uxy, L.uz, ct, unit_open(C.draw(L)));
}

// The end of a step: score an exit, or play roulette (physics.hpp:250-259); the step cap; publish
// an ended packet (unless the kernel does: Ctx::kPublishAtRelaunch). Returns true when the packet
// has ended.
template <int FAST, class Ctx> __device__ __forceinline__ bool step_tail(Lane &L, Ctx &C, int exit_kind, bool died) {
    // one test on the common path for the three rare ends of a step: an exit, a weight below the
    // roulette threshold, the step cap (measured 0.4 % faster on skin5 than three tests)
    if (exit_kind != 0 || L.w < kWeightMin || L.steps >= C.step_cap) {
        if (exit_kind) {
            // ---- score the exit (check, totals, R_d(r,a) or T_t(r,a))
            const float n2 = norm2(L.uxy, L.uz);
            if (!(L.w == L.w) || !(fabsf(fsub(n2, 1.0f)) <= 1e-5f)) ++L.anomalies;
            const unsigned long long v = to_fixed(L.w);
            C.batch_add(L, exit_kind - 1, v);
            C.exit(L, exit_kind, v);
        } else if (L.w < kWeightMin) {
            // ---- roulette (physics.hpp:250-259)
            if (L.w == 0.0f) {
                died = true;
            } else if (unit_open(C.draw(L)) < kChance) {
                if constexpr (Math<FAST>::div) L.w = fmul(L.w, 10.0f);
                else L.w /= kChance;
            } else {
                died = true;
            }
        }
        if (!died && L.steps >= C.step_cap) {  // a packet that never ends is an anomaly, not a hang
            ++L.anomalies;
            died = true;
        }
    }
    if constexpr (!Ctx::kPublishAtRelaunch) {
        if (died) finish_photon(L, C);
    }
    return died;
}

// One hop-drop-spin (or boundary) step plus roulette (step_once, physics.hpp:263-277); returns true
// when the packet has ended. Its per-photon totals are then published here, or, when the context
// says Ctx::kPublishAtRelaunch, by the kernel when the lane takes its next photon or runs out (one
// warp-uniform place instead of a branch in every step).
template <int FAST, class Ctx> __device__ __forceinline__ bool walk_step(Lane &L, Ctx &C) {
    bool died = false;
    int exit_kind = 0;
    const Hot h = hot_of(L, C);
    if (step_move<FAST>(L, C, h)) step_boundary<FAST>(L, C, exit_kind, died);
    else step_interaction<FAST>(L, C, h);
    return step_tail<FAST>(L, C, exit_kind, died);
}

// This lane's slot 0 in its block's ring area: each warp has its own region of kRingWords slots,
// slot k of its 32 lanes contiguous, so the lanes of a warp never conflict on a bank.
__device__ __forceinline__ int ring_lane_offset() {
    return static_cast<int>((threadIdx.x >> 5) * (kRingWords * 32u) + (threadIdx.x & 31u));
}

// The random-word ring: kRingWords words per lane in shared memory.
struct Ring {
    uint32_t *base;  // this lane's slot 0 (ring_lane_offset)

    __device__ __forceinline__ uint32_t draw(Lane &L) const {
        const uint32_t o = base[(L.rp & (kRingWords - 1u)) * slot_stride()];
        ++L.rp;
        return o;
    }
    // pass over the next word without reading it
    __device__ __forceinline__ void skip(Lane &L) const { ++L.rp; }
    // read the next word without passing over it
    __device__ __forceinline__ uint32_t peek(const Lane &L) const { return base[(L.rp & (kRingWords - 1u)) * slot_stride()]; }
    // each warp's ring is its own region: slot k of its 32 lanes at k * 32 words (a constant stride:
    // the slot addresses take shifts instead of multiplications)
    __device__ __forceinline__ static constexpr int slot_stride() { return 32; }
    __device__ __forceinline__ void store(Lane &L, uint32_t b0, uint32_t b1, uint32_t b2, uint32_t b3) const {
        ++L.blk;
        uint32_t *const slot = base + (L.wp & (kRingWords - 4u)) * slot_stride();  // wp is a multiple of 4
        slot[0] = b0;
        slot[slot_stride()] = b1;
        slot[2 * slot_stride()] = b2;
        slot[3 * slot_stride()] = b3;
        L.wp += 4u;
    }
    __device__ __forceinline__ void refill(Lane &L, uint32_t k0, uint32_t k1) const {
        uint32_t b0, b1, b2, b3;
        philox4x32_10(L.id, 0u, L.blk, k0, k1, b0, b1, b2, b3);
        store(L, b0, b1, b2, b3);
    }
    // with a precomputed key schedule (one key for every lane of the launch)
    __device__ __forceinline__ void refill(Lane &L, const uint32_t (&rk)[20]) const {
        uint32_t b0, b1, b2, b3;
        philox4x32_10_rk(L.id, 0u, L.blk, rk, b0, b1, b2, b3);
        store(L, b0, b1, b2, b3);
    }
    // with this lane's key schedule in shared memory (key_schedule_store)
    __device__ __forceinline__ void refill(Lane &L, const uint4 *sched, int sched_stride) const {
        uint32_t b0, b1, b2, b3;
        philox4x32_10_sched(L.id, 0u, L.blk, sched, sched_stride, b0, b1, b2, b3);
        store(L, b0, b1, b2, b3);
    }
};

}  // namespace tmc
