// The persistent photon-walk kernel (see walk.cuh for the design and the reference citations).
#pragma once

#include "walk.cuh"

namespace tmc {

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
    h.mua = L.mua;
    h.mut = L.mut;
    h.inv_mut = L.inv_mut;
    h.absorb = L.absorb;
    h.z0 = L.z0;
    h.z1 = L.z1;
    h.g = L.g;
    h.hg_a = L.hg_a;
    h.hg_b = L.hg_b;
    h.hg_c = L.hg_c;
    h.hg_d = L.hg_d;
    h.inv_2g = L.inv_2g;
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
    const float sa1 = m_sqrt<FAST>(1.0f - ca1 * ca1);
    float sa2;
    if constexpr (Math<FAST>::div) sa2 = sa1 * rat;
    else sa2 = n1 * sa1 / n2;
    if (sa2 >= 1.0f) {
        ca2 = 0.0f;
        return 1.0f;
    }
    ca2 = m_sqrt<FAST>(1.0f - sa2 * sa2);
    const float cap = ca1 * ca2 - sa1 * sa2;
    const float cam = ca1 * ca2 + sa1 * sa2;
    const float sap = sa1 * ca2 + ca1 * sa2;
    const float sam = sa1 * ca2 - ca1 * sa2;
    return m_div<FAST>(0.5f * sam * sam * (cam * cam + cap * cap), sap * sap * cam * cam);
}

template <int FAST> __device__ __forceinline__ int bin_of(float x, float width, float inv_width, int n) {
    if constexpr (Math<FAST>::div) {
        return clamp_bin(x, inv_width, n);
    } else {
        if (!(x > 0.0f)) return 0;
        const float i = x / width;
        return i >= static_cast<float>(n) ? n - 1 : static_cast<int>(i);
    }
}

// Shared-memory layout of one block, in 64-bit words (offsets computed identically on the host).
struct SmemLayout {
    int batch, core_a, lastz_a, lastr_a, rd, tt, layers, total;  // word offsets / total words
};

__host__ __device__ inline SmemLayout smem_layout(const WalkParams &P) {
    SmemLayout s;
    int off = 0;
    s.batch = off;
    off += P.batch_smem ? P.nb * (4 + P.nl) : 0;
    s.core_a = off;
    off += P.tr_a * P.tz_a;
    // The clamped last depth bin and last radius bin of A(r,z) collect every deposit beyond the
    // grid; for a deep or wide stack they are the hottest bins, so a tile that does not cover the
    // whole grid always carries them too (a "cross": core + last column + last row).
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

template <int FAST>
__global__ void __launch_bounds__(256) walk_kernel(const __grid_constant__ WalkParams P) {
    extern __shared__ __align__(16) unsigned long long smem[];
    const SmemLayout S = smem_layout(P);
    const int bstride = 4 + P.nl;
    for (int i = threadIdx.x; i < S.layers; i += blockDim.x) smem[i] = 0ull;
    {
        const float *src = reinterpret_cast<const float *>(P.layers);
        float *dst = reinterpret_cast<float *>(smem + S.layers);
        for (int i = threadIdx.x; i < P.nl * static_cast<int>(sizeof(LayerC) / 4); i += blockDim.x) dst[i] = src[i];
    }
    __syncthreads();
    const LayerC *s_layers = reinterpret_cast<const LayerC *>(smem + S.layers);
    unsigned long long *const bt = P.batch_smem ? smem + S.batch : P.g_batch;
    unsigned long long *const s_core = smem + S.core_a;
    unsigned long long *const s_lastz = smem + S.lastz_a;
    unsigned long long *const s_lastr = smem + S.lastr_a;
    unsigned long long *const s_rd = smem + S.rd;
    unsigned long long *const s_tt = smem + S.tt;
    const bool cross = P.profiles && P.cross;

    const unsigned lane = threadIdx.x & 31u;
    const unsigned lt_mask = (1u << lane) - 1u;
    const uint32_t k0 = static_cast<uint32_t>(P.seed), k1 = static_cast<uint32_t>(P.seed >> 32);

    unsigned long long pool_next = 0ull, pool_end = 0ull;  // warp-uniform photon-id pool
    bool alive = false, exhausted = false;

    float x = 0.f, y = 0.f, z = 0.f, ux = 0.f, uy = 0.f, uz = 1.f, w = 0.f, sleft = 0.f;
    int layer = 0, batch = 0;
    uint32_t id_lo = 0u, id_hi = 0u, blk = 0u;
    uint32_t q0 = 0u, q1 = 0u, q2 = 0u, q3 = 0u, q4 = 0u, q5 = 0u, q6 = 0u;
    int nq = 0;
    uint32_t events = 0u, anomalies = 0u, steps = 0u;
    unsigned long long run_abs = 0ull;   // fixed-point weight absorbed in the current layer
    int cache_bin = -1;                  // one-entry run cache of A(r,z) deposits (global index)
    unsigned long long cache_val = 0ull;
    Hot h;
    load_hot(h, s_layers[0]);

    auto draw = [&]() -> uint32_t {
        const uint32_t o = q0;
        q0 = q1;
        q1 = q2;
        q2 = q3;
        q3 = q4;
        q4 = q5;
        q5 = q6;
        --nq;
        return o;
    };

    // Deposit into A(r,z) at global bin (ir, iz).
    auto deposit = [&](int ir, int iz, unsigned long long v) {
        if (ir < P.tr_a && iz < P.tz_a) {
            atomicAdd(&s_core[ir * P.tz_a + iz], v);
        } else if (cross && iz == P.nz - 1) {
            atomicAdd(&s_lastz[ir], v);
        } else if (cross && ir == P.nr - 1) {
            atomicAdd(&s_lastr[iz], v);
        } else {
            atomicAdd(&P.g_arz[static_cast<size_t>(ir) * P.nz + iz], v);
        }
    };

    for (;;) {
        // ---- relaunch: lanes without a photon take the next ids from the warp's pool
        const unsigned need = __ballot_sync(0xffffffffu, !alive && !exhausted);
        if (need) {
            const unsigned n = __popc(need);
            const unsigned rank = __popc(need & lt_mask);
            const unsigned long long avail = pool_end - pool_next;
            unsigned long long my;
            if (avail >= n) {
                my = pool_next + rank;
                pool_next += n;
            } else {
                const int leader = __ffs(need) - 1;
                unsigned long long base = 0ull;
                if (static_cast<int>(lane) == leader)
                    base = atomicAdd(P.counter, static_cast<unsigned long long>(P.chunk));
                base = __shfl_sync(0xffffffffu, base, leader);
                my = rank < avail ? pool_next + rank : base + (rank - avail);
                pool_next = base + (n - avail);
                pool_end = base + static_cast<unsigned long long>(P.chunk);
            }
            if (!alive && !exhausted) {
                if (my >= P.photons) {
                    exhausted = true;
                } else {
                    // launch (physics.hpp:58-66) and the photon's own stream (seed, id)
                    id_lo = static_cast<uint32_t>(my);
                    id_hi = static_cast<uint32_t>(my >> 32);
                    blk = 0u;
                    nq = 0;
                    x = y = z = 0.f;
                    ux = uy = 0.f;
                    uz = 1.f;
                    w = P.launch_w;
                    sleft = 0.f;
                    if (layer != 0) {
                        layer = 0;
                        load_hot(h, s_layers[0]);
                    }
                    const unsigned long long bnd = P.plan_extra * (P.plan_base + 1ull);
                    batch = static_cast<int>(my < bnd ? my / (P.plan_base + 1ull)
                                                      : P.plan_extra + (my - bnd) / P.plan_base);
                    events = anomalies = steps = 0u;
                    run_abs = 0ull;
                    alive = true;
                }
            }
        }
        if (!__any_sync(0xffffffffu, alive)) break;
        if (!alive) continue;

        // ---- one step (physics.hpp:263-277)
        if (nq < 4) {  // a step draws at most 4 words; keep the stream's order exactly
            uint32_t b0, b1, b2, b3;
            philox4x32_10(id_lo, id_hi, blk, k0, k1, b0, b1, b2, b3);
            ++blk;
            if (nq == 0) {
                q0 = b0; q1 = b1; q2 = b2; q3 = b3;
            } else if (nq == 1) {
                q1 = b0; q2 = b1; q3 = b2; q4 = b3;
            } else if (nq == 2) {
                q2 = b0; q3 = b1; q4 = b2; q5 = b3;
            } else {
                q3 = b0; q4 = b1; q5 = b2; q6 = b3;
            }
            nq += 4;
        }
        ++steps;
        float s;
        if (sleft == 0.0f) {
            const float u = unit_open(draw());
            if constexpr (Math<FAST>::log) {
                // the SFU logarithm's absolute error can flip the sign of log(u) for the two
                // largest u of the 23-bit grid; a step is never negative
                s = fmaxf(-m_log<FAST>(u), 0.0f) * h.inv_mut;
            } else if constexpr (Math<FAST>::div) {
                s = -m_log<FAST>(u) * h.inv_mut;
            } else {
                s = -m_log<FAST>(u) / h.mut;
            }
        } else {
            if constexpr (Math<FAST>::div) s = sleft * h.inv_mut;
            else s = sleft / h.mut;
            sleft = 0.0f;
        }
        bool hit = false;
        if (uz != 0.0f) {
            const float db = m_div<FAST>((uz > 0.0f ? h.z1 : h.z0) - z, uz);
            if (s > db) {
                sleft = (s - db) * h.mut;
                s = db;
                hit = true;
            }
        }
        x += s * ux;
        y += s * uy;
        z += s * uz;

        bool died = false;
        int exit_kind = 0;  // 1: reflectance (top), 2: transmittance (bottom)
        if (hit) {
            // ---- boundary: reflect, or transmit into the next layer or out (physics.hpp:198-246)
            const LayerC &Lc = s_layers[layer];
            const bool up = uz < 0.0f;
            const float ca1 = up ? -uz : uz;
            const float nt = up ? Lc.n_up : Lc.n_dn;
            const float rat = up ? Lc.rat_up : Lc.rat_dn;
            float uz1 = 0.0f;
            const float r = (ca1 <= (up ? Lc.cc_up : Lc.cc_dn))
                                ? 1.0f
                                : fresnel<FAST>(Lc.n, nt, ca1, up ? Lc.rn_up : Lc.rn_dn, rat, uz1);
            if (unit_open(draw()) > r) {
                ux *= rat;
                uy *= rat;
                uz = up ? -uz1 : uz1;
                if (up ? layer == 0 : layer == P.nl - 1) {
                    exit_kind = up ? 1 : 2;
                    died = true;
                } else {
                    if (run_abs) {
                        atomicAdd(&bt[batch * bstride + 4 + layer], run_abs);
                        run_abs = 0ull;
                    }
                    layer += up ? -1 : 1;
                    load_hot(h, s_layers[layer]);
                }
            } else {
                uz = -uz;
            }
        } else {
            // ---- drop (physics.hpp:187-193) and score the absorption
            float dwa;
            if constexpr (Math<FAST>::div) dwa = w * h.absorb;
            else dwa = w * h.mua / h.mut;
            w -= dwa;
            ++events;
            {
                const float n2 = ux * ux + uy * uy + uz * uz;
                if (!(dwa == dwa) || !(fabsf(n2 - 1.0f) <= 1e-5f)) ++anomalies;
            }
            const unsigned long long v = to_fixed(dwa);
            run_abs += v;
            if (P.profiles) {
                const float r2 = x * x + y * y;
                const float rr = r2 > 0.0f ? m_sqrt<FAST>(r2) : 0.0f;
                const int ir = bin_of<FAST>(rr, P.dr, P.inv_dr, P.nr);
                const int iz = bin_of<FAST>(z, P.dz, P.inv_dz, P.nz);
                const int key = ir * P.nz + iz;
                if (key == cache_bin) {
                    cache_val += v;
                } else {
                    if (cache_bin >= 0) deposit(cache_bin / P.nz, cache_bin % P.nz, cache_val);
                    cache_bin = key;
                    cache_val = v;
                }
            }
            // ---- spin (physics.hpp:101-144)
            float ct;
            {
                const float xi = unit_open(draw());
                if (h.g == 0.0f) {
                    ct = 2.0f * xi - 1.0f;
                } else {
                    const float t = m_div<FAST>(h.hg_a, h.hg_b + h.hg_c * xi);
                    if constexpr (Math<FAST>::div) ct = (h.hg_d - t * t) * h.inv_2g;
                    else ct = (h.hg_d - t * t) / h.hg_c;
                    ct = fminf(fmaxf(ct, -1.0f), 1.0f);
                }
            }
            float st = 1.0f - ct * ct;
            st = st > 0.0f ? m_sqrt<FAST>(st) : 0.0f;
            float sp, cp;
            {
                const float u = unit_open(draw());
                if constexpr (Math<FAST>::sincos) {
                    // psi - pi lies in (-pi, pi), where the SFU sine and cosine are accurate
                    __sincosf(kTwoPi * (u - 0.5f), &sp, &cp);
                    sp = -sp;
                    cp = -cp;
                } else {
                    sincosf(kTwoPi * u, &sp, &cp);
                }
            }
            if (fabsf(uz) > kCosZero) {
                ux = st * cp;
                uy = st * sp;
                uz = uz >= 0.0f ? ct : -ct;
            } else {
                const float ox = ux, oy = uy, oz = uz;
                if constexpr (Math<FAST>::sqrt) {
                    const float it = rsqrtf(1.0f - oz * oz);
                    ux = st * (ox * oz * cp - oy * sp) * it + ox * ct;
                    uy = st * (oy * oz * cp + ox * sp) * it + oy * ct;
                    uz = -st * cp * (1.0f - oz * oz) * it + oz * ct;
                } else {
                    const float tmp = sqrtf(1.0f - oz * oz);
                    ux = st * (ox * oz * cp - oy * sp) / tmp + ox * ct;
                    uy = st * (oy * oz * cp + ox * sp) / tmp + oy * ct;
                    uz = -st * cp * tmp + oz * ct;
                }
            }
            const float inv = m_rsqrt<FAST>(ux * ux + uy * uy + uz * uz);
            ux *= inv;
            uy *= inv;
            uz *= inv;
        }

        if (exit_kind) {
            // ---- score the exit (check, totals, R_d(r,a) or T_t(r,a))
            const float n2 = ux * ux + uy * uy + uz * uz;
            if (!(w == w) || !(fabsf(n2 - 1.0f) <= 1e-5f)) ++anomalies;
            const unsigned long long v = to_fixed(w);
            atomicAdd(&bt[batch * bstride + (exit_kind - 1)], v);
            if (P.profiles) {
                const float r2 = x * x + y * y;
                const float rr = r2 > 0.0f ? m_sqrt<FAST>(r2) : 0.0f;
                const int ir = bin_of<FAST>(rr, P.dr, P.inv_dr, P.nr);
                const int ia = bin_of<FAST>(acosf(fminf(fabsf(uz), 1.0f)), P.da, P.inv_da, P.na);
                if (exit_kind == 1) {
                    if (ir < P.tr_rd) atomicAdd(&s_rd[ir * P.na + ia], v);
                    else atomicAdd(&P.g_rd[ir * P.na + ia], v);
                } else {
                    if (ir < P.tr_tt) atomicAdd(&s_tt[ir * P.na + ia], v);
                    else atomicAdd(&P.g_tt[ir * P.na + ia], v);
                }
            }
        } else if (w < kWeightMin) {
            // ---- roulette (physics.hpp:250-259)
            if (w == 0.0f) {
                died = true;
            } else if (unit_open(draw()) < kChance) {
                if constexpr (Math<FAST>::div) w *= 10.0f;
                else w /= kChance;
            } else {
                died = true;
            }
        }
        if (!died && steps >= P.step_cap) {  // a packet that never ends is an anomaly, not a hang
            ++anomalies;
            died = true;
        }
        if (died) {
            const int base = batch * bstride;
            atomicAdd(&bt[base + 2], static_cast<unsigned long long>(events));
            if (anomalies) atomicAdd(&bt[base + 3], static_cast<unsigned long long>(anomalies));
            if (run_abs) atomicAdd(&bt[base + 4 + layer], run_abs);
            if (cache_bin >= 0) {
                deposit(cache_bin / P.nz, cache_bin % P.nz, cache_val);
                cache_bin = -1;
                cache_val = 0ull;
            }
            alive = false;
        }
    }

    // ---- publish the block's shared tallies into the global ones (integer adds: exact)
    __syncthreads();
    if (P.batch_smem) {
        for (int i = threadIdx.x; i < P.nb * bstride; i += blockDim.x) {
            const unsigned long long v = smem[S.batch + i];
            if (v) atomicAdd(&P.g_batch[i], v);
        }
    }
    for (int i = threadIdx.x; i < P.tr_a * P.tz_a; i += blockDim.x) {
        const unsigned long long v = s_core[i];
        if (v) atomicAdd(&P.g_arz[static_cast<size_t>(i / P.tz_a) * P.nz + (i % P.tz_a)], v);
    }
    if (cross) {
        for (int i = threadIdx.x; i < P.nr; i += blockDim.x) {
            const unsigned long long v = s_lastz[i];
            if (v) atomicAdd(&P.g_arz[static_cast<size_t>(i) * P.nz + (P.nz - 1)], v);
        }
        for (int i = threadIdx.x; i < P.nz; i += blockDim.x) {
            const unsigned long long v = s_lastr[i];
            if (v) atomicAdd(&P.g_arz[static_cast<size_t>(P.nr - 1) * P.nz + i], v);
        }
    }
    for (int i = threadIdx.x; i < P.tr_rd * P.na; i += blockDim.x) {
        const unsigned long long v = s_rd[i];
        if (v) atomicAdd(&P.g_rd[i], v);
    }
    for (int i = threadIdx.x; i < P.tr_tt * P.na; i += blockDim.x) {
        const unsigned long long v = s_tt[i];
        if (v) atomicAdd(&P.g_tt[i], v);
    }
}

}  // namespace tmc
