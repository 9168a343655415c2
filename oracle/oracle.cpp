// ORACLE — test infrastructure only. Nothing in the product (the tissuemc_b200 package, its CUDA
// kernels, its C ABI or its CLI) links, loads or calls this file. Only tests/, the smoke check in
// __graft_entry__.py and the cpu_baseline leg of bench.py use it, and only as the checker.
//
// A CPU restatement of TissueMC's MCML photon walk and of its CPU engine, written from the
// reference's sources as a specification (paths are relative to the TissueMC project root):
//
//   Philox4x32-10 and the per-photon stream ......... include/tissuemc/philox.hpp:49-57, 62-83, 127-140
//   launch / specular reflectance .................... include/tissuemc/physics.hpp:50-66
//   Fresnel reflectance .............................. include/tissuemc/physics.hpp:71-98
//   Henyey-Greenstein sampling and spin .............. include/tissuemc/physics.hpp:101-144
//   step size, boundary distance, hop, drop .......... include/tissuemc/physics.hpp:148-193
//   boundary crossing, roulette, step_once ........... include/tissuemc/physics.hpp:198-287
//   layer geometry and critical cosines .............. include/tissuemc/config.hpp:70-101
//   batch plan ....................................... include/tissuemc/batching.hpp:11-29
//   Neumaier compensated sum ......................... include/tissuemc/accumulate.hpp:15-30
//   CPU tally, bin clamp, anomaly check, batch loop .. src/cpu/engine.cpp:22-115
//   worker pool and in-order batch merge ............. src/cpu/engine.cpp:119-214
//
// On top of the reference's tallies (per-batch R_d, T_t, absorbed per layer, events, anomalies,
// and the 1-D profiles A(z), R_d(r)) it adds the 2-D tallies the reference does not have:
// A(r,z), R_d(r,a), T_t(r,a), with the MCML binning ir = floor(r/dr), iz = floor(z/dz),
// ia = floor(acos(|uz_exit|) / (pi / (2 na))), each clamped to the last bin, and a per-bin count
// of contributing scores. The reference's own 1-D projections are computed exactly as it computes
// them, so on the same run they must equal its a_z and rd_r bit for bit (tests check this against
// outputs of the reference binary).
//
// Arithmetic is written in the same order as the reference so that, compiled by g++ for x86-64
// without -ffast-math or FMA contraction, float64 and float32 transport reproduce the reference
// CPU engine's results exactly.

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <exception>
#include <mutex>
#include <thread>
#include <vector>

namespace oracle {

// ---------------------------------------------------------------- Philox4x32-10 (Salmon et al.)
struct Block {
    uint32_t v[4];
};

static inline Block philox_round(const Block &c, uint32_t k0, uint32_t k1) {
    const uint64_t p0 = static_cast<uint64_t>(0xD2511F53u) * c.v[0];
    const uint64_t p1 = static_cast<uint64_t>(0xCD9E8D57u) * c.v[2];
    Block o;
    o.v[0] = static_cast<uint32_t>(p1 >> 32) ^ c.v[1] ^ k0;
    o.v[1] = static_cast<uint32_t>(p1);
    o.v[2] = static_cast<uint32_t>(p0 >> 32) ^ c.v[3] ^ k1;
    o.v[3] = static_cast<uint32_t>(p0);
    return o;
}

static inline Block philox10(Block c, uint32_t k0, uint32_t k1) {
    c = philox_round(c, k0, k1);
    for (int r = 1; r < 10; ++r) {
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
        c = philox_round(c, k0, k1);
    }
    return c;
}

// One photon's stream: counter = {id lo, id hi, block index, 0}, key = 64-bit seed.
struct Stream {
    uint32_t c0, c1, blk, k0, k1;
    Block buf;
    int used;
    Stream(uint64_t seed, uint64_t id)
        : c0(static_cast<uint32_t>(id)), c1(static_cast<uint32_t>(id >> 32)), blk(0),
          k0(static_cast<uint32_t>(seed)), k1(static_cast<uint32_t>(seed >> 32)), buf{}, used(4) {}
    uint32_t word() {
        if (used == 4) {
            buf = philox10(Block{{c0, c1, blk, 0u}}, k0, k1);
            ++blk;
            used = 0;
        }
        return buf.v[used++];
    }
};

template <class Real> Real open01(uint32_t x);
template <> inline double open01<double>(uint32_t x) { return (static_cast<double>(x) + 0.5) * 0x1p-32; }
template <> inline float open01<float>(uint32_t x) { return (static_cast<float>(x >> 9) + 0.5f) * 0x1p-23f; }

template <class Real> inline Real draw(Stream &s) { return open01<Real>(s.word()); }

// ---------------------------------------------------------------- constants and geometry
template <class Real> struct K;
template <> struct K<double> {
    static constexpr double pi = 3.14159265358979323846, wmin = 1e-4, chance = 0.1,
                            cos_zero = 1.0 - 1e-12, cos_90 = 1e-6;
};
template <> struct K<float> {
    static constexpr float pi = 3.14159265358979323846f, wmin = 1e-4f, chance = 0.1f,
                           cos_zero = 1.0f - 1e-6f, cos_90 = 1e-6f;
};

constexpr int kMaxLayers = 16;

template <class Real> struct Slab {
    Real n, mua, mus, g, z0, z1, cc_top, cc_bot;
};

template <class Real> struct Geo {
    int nl;
    Real n_above, n_below;
    Slab<Real> L[kMaxLayers];
    Real dz, dr;
    int nz, nr, na;
};

}  // namespace oracle

extern "C" {
// Input description; mirrors one parsed .mci run (src/io/mci.cpp:97-171 of the reference).
typedef struct {
    double n, mua, mus, g, d;
} oracle_layer;

typedef struct {
    double dz, dr;
    int32_t nz, nr, na;
    double n_above, n_below;
    int32_t num_layers;
    oracle_layer layers[16];
} oracle_spec;

// Caller-allocated outputs. Pointers marked optional may be NULL.
typedef struct {
    double *rd, *tt;              // [B]
    double *absorbed;             // [B * L]
    uint64_t *events, *anomalies; // [B]
    double *a_z, *rd_r;           // [nz], [nr]      merged exactly as the reference merges them
    double *a_rz;                 // [nr * nz]       r-major, as MCML's A_rz[ir][iz]
    double *rd_ra, *tt_ra;        // [nr * na]
    uint64_t *n_a_rz;             // optional [nr * nz]  scores per bin
    uint64_t *n_rd_ra, *n_tt_ra;  // optional [nr * na]
    double *b_a_rz;               // optional [B * nr * nz]  per-batch bins (for standard errors)
    double *b_rd_ra, *b_tt_ra;    // optional [B * nr * na]
    uint64_t *boundary_steps;     // optional [B]  steps that ended on a layer boundary
    double specular;
    double wall_seconds;
    int32_t threads_used;
    char error[256];
} oracle_out;
}

namespace oracle {

struct Neumaier {
    double s = 0, c = 0;
    void add(double x) {
        const double t = s + x;
        if (std::fabs(s) >= std::fabs(x)) {
            c += (s - t) + x;
        } else {
            c += (x - t) + s;
        }
        s = t;
    }
    double value() const { return s + c; }
};

static double crit_cos(double ni, double nt) { return ni > nt ? std::sqrt(1.0 - (nt * nt) / (ni * ni)) : 0.0; }

template <class Real> Geo<Real> make_geo(const oracle_spec &sp) {
    Geo<Real> g{};
    g.nl = sp.num_layers;
    g.n_above = static_cast<Real>(sp.n_above);
    g.n_below = static_cast<Real>(sp.n_below);
    double z = 0.0;
    for (int i = 0; i < sp.num_layers; ++i) {
        const oracle_layer &s = sp.layers[i];
        const double nt = i == 0 ? sp.n_above : sp.layers[i - 1].n;
        const double nb = i + 1 == sp.num_layers ? sp.n_below : sp.layers[i + 1].n;
        Slab<Real> &L = g.L[i];
        L.n = static_cast<Real>(s.n);
        L.mua = static_cast<Real>(s.mua);
        L.mus = static_cast<Real>(s.mus);
        L.g = static_cast<Real>(s.g);
        L.z0 = static_cast<Real>(z);
        z += s.d;
        L.z1 = static_cast<Real>(z);
        L.cc_top = static_cast<Real>(crit_cos(s.n, nt));
        L.cc_bot = static_cast<Real>(crit_cos(s.n, nb));
    }
    g.dz = static_cast<Real>(sp.dz);
    g.dr = static_cast<Real>(sp.dr);
    g.nz = sp.nz;
    g.nr = sp.nr;
    g.na = sp.na;
    return g;
}

template <class Real> Real specular(const Geo<Real> &g) {
    const Real n0 = g.n_above, n1 = g.L[0].n;
    const Real r = (n0 - n1) / (n0 + n1);
    return r * r;
}

template <class Real> struct Packet {
    Real x, y, z, ux, uy, uz, w, s, sleft;
    int layer;
    bool dead;
};

// Reference src/cpu/engine.cpp:59-66: clamp at both ends.
static inline size_t clamp_bin(double x, double width, int count) {
    if (!(x > 0)) {
        return 0;
    }
    const double i = x / width;
    return i >= static_cast<double>(count) ? static_cast<size_t>(count - 1) : static_cast<size_t>(i);
}

// Per-batch tally (reference CpuTally, src/cpu/engine.cpp:22-90) plus the 2-D arrays.
template <class Real> struct BatchTally {
    const Geo<Real> &g;
    Neumaier rd, tt;
    std::vector<Neumaier> absorbed, az, rr, arz, rra, tra;
    std::vector<uint64_t> n_arz, n_rra, n_tra;
    uint64_t events = 0, anomalies = 0, boundary = 0;
    bool counts;
    double da;

    BatchTally(const Geo<Real> &geo, bool want_counts)
        : g(geo), absorbed(geo.nl), az(geo.nz), rr(geo.nr),
          arz(static_cast<size_t>(geo.nr) * geo.nz), rra(static_cast<size_t>(geo.nr) * geo.na),
          tra(static_cast<size_t>(geo.nr) * geo.na), counts(want_counts),
          da(0.5 * 3.14159265358979323846 / geo.na) {
        if (counts) {
            n_arz.assign(arz.size(), 0);
            n_rra.assign(rra.size(), 0);
            n_tra.assign(tra.size(), 0);
        }
    }

    void check(const Packet<Real> &p, Real w) {
        constexpr double tol = sizeof(Real) == sizeof(double) ? 1e-9 : 1e-5;
        const double ux = p.ux, uy = p.uy, uz = p.uz;
        const double n2 = ux * ux + uy * uy + uz * uz;
        if (!std::isfinite(static_cast<double>(w)) || !std::isfinite(n2) || std::fabs(n2 - 1.0) > tol) {
            ++anomalies;
        }
    }

    size_t rbin(const Packet<Real> &p) const {
        const double r = std::sqrt(static_cast<double>(p.x) * static_cast<double>(p.x) +
                                   static_cast<double>(p.y) * static_cast<double>(p.y));
        return clamp_bin(r, static_cast<double>(g.dr), g.nr);
    }

    size_t abin(const Packet<Real> &p) const {
        return clamp_bin(std::acos(std::fabs(static_cast<double>(p.uz))), da, g.na);
    }

    void absorb(const Packet<Real> &p, Real w) {
        ++events;
        check(p, w);
        absorbed[static_cast<size_t>(p.layer)].add(static_cast<double>(w));
        const size_t iz = clamp_bin(static_cast<double>(p.z), static_cast<double>(g.dz), g.nz);
        az[iz].add(static_cast<double>(w));
        const size_t k = rbin(p) * static_cast<size_t>(g.nz) + iz;
        arz[k].add(static_cast<double>(w));
        if (counts) {
            ++n_arz[k];
        }
    }

    void reflect(const Packet<Real> &p, Real w) {
        check(p, w);
        rd.add(static_cast<double>(w));
        const size_t ir = rbin(p);
        rr[ir].add(static_cast<double>(w));
        const size_t k = ir * static_cast<size_t>(g.na) + abin(p);
        rra[k].add(static_cast<double>(w));
        if (counts) {
            ++n_rra[k];
        }
    }

    void transmit(const Packet<Real> &p, Real w) {
        check(p, w);
        tt.add(static_cast<double>(w));
        const size_t k = rbin(p) * static_cast<size_t>(g.na) + abin(p);
        tra[k].add(static_cast<double>(w));
        if (counts) {
            ++n_tra[k];
        }
    }
};

// ---------------------------------------------------------------- the walk (physics.hpp:50-287)
template <class Real> Real fresnel_r(Real n1, Real n2, Real ca1, Real &ca2) {
    using C = K<Real>;
    if (n1 == n2) {
        ca2 = ca1;
        return Real(0);
    }
    if (ca1 > C::cos_zero) {
        ca2 = ca1;
        const Real r = (n2 - n1) / (n2 + n1);
        return r * r;
    }
    if (ca1 < C::cos_90) {
        ca2 = Real(0);
        return Real(1);
    }
    const Real sa1 = std::sqrt(Real(1) - ca1 * ca1);
    const Real sa2 = n1 * sa1 / n2;
    if (sa2 >= Real(1)) {
        ca2 = Real(0);
        return Real(1);
    }
    ca2 = std::sqrt(Real(1) - sa2 * sa2);
    const Real cap = ca1 * ca2 - sa1 * sa2;
    const Real cam = ca1 * ca2 + sa1 * sa2;
    const Real sap = sa1 * ca2 + ca1 * sa2;
    const Real sam = sa1 * ca2 - ca1 * sa2;
    return Real(0.5) * sam * sam * (cam * cam + cap * cap) / (sap * sap * cam * cam);
}

template <class Real> Real hg_cos(Real gg, Stream &rng) {
    const Real xi = draw<Real>(rng);
    if (gg == Real(0)) {
        return Real(2) * xi - Real(1);
    }
    const Real t = (Real(1) - gg * gg) / (Real(1) - gg + Real(2) * gg * xi);
    Real c = (Real(1) + gg * gg - t * t) / (Real(2) * gg);
    if (c < Real(-1)) c = Real(-1);
    if (c > Real(1)) c = Real(1);
    return c;
}

template <class Real> void scatter(Packet<Real> &p, Real gg, Stream &rng) {
    using C = K<Real>;
    const Real ct = hg_cos(gg, rng);
    Real st = Real(1) - ct * ct;
    st = st > Real(0) ? std::sqrt(st) : Real(0);
    const Real psi = Real(2) * C::pi * draw<Real>(rng);
    const Real cp = std::cos(psi);
    const Real sp = std::sin(psi);
    if (std::fabs(p.uz) > C::cos_zero) {
        p.ux = st * cp;
        p.uy = st * sp;
        p.uz = p.uz >= Real(0) ? ct : -ct;
    } else {
        const Real tmp = std::sqrt(Real(1) - p.uz * p.uz);
        const Real ux = p.ux, uy = p.uy, uz = p.uz;
        p.ux = st * (ux * uz * cp - uy * sp) / tmp + ux * ct;
        p.uy = st * (uy * uz * cp + ux * sp) / tmp + uy * ct;
        p.uz = -st * cp * tmp + uz * ct;
    }
    const Real inv = Real(1) / std::sqrt(p.ux * p.ux + p.uy * p.uy + p.uz * p.uz);
    p.ux *= inv;
    p.uy *= inv;
    p.uz *= inv;
}

template <class Real> void cross(Packet<Real> &p, const Geo<Real> &g, Stream &rng, BatchTally<Real> &t) {
    const Slab<Real> &L = g.L[p.layer];
    const Real ni = L.n;
    Real uz1 = Real(0);
    Real r;
    if (p.uz < Real(0)) {
        const Real nt = p.layer == 0 ? g.n_above : g.L[p.layer - 1].n;
        r = (-p.uz <= L.cc_top) ? Real(1) : fresnel_r(ni, nt, -p.uz, uz1);
        if (draw<Real>(rng) > r) {
            p.ux *= ni / nt;
            p.uy *= ni / nt;
            p.uz = -uz1;
            if (p.layer == 0) {
                t.reflect(p, p.w);
                p.dead = true;
            } else {
                --p.layer;
            }
        } else {
            p.uz = -p.uz;
        }
    } else {
        const bool last = p.layer == g.nl - 1;
        const Real nt = last ? g.n_below : g.L[p.layer + 1].n;
        r = (p.uz <= L.cc_bot) ? Real(1) : fresnel_r(ni, nt, p.uz, uz1);
        if (draw<Real>(rng) > r) {
            p.ux *= ni / nt;
            p.uy *= ni / nt;
            p.uz = uz1;
            if (last) {
                t.transmit(p, p.w);
                p.dead = true;
            } else {
                ++p.layer;
            }
        } else {
            p.uz = -p.uz;
        }
    }
}

template <class Real> void one_step(Packet<Real> &p, const Geo<Real> &g, Stream &rng, BatchTally<Real> &t) {
    const Slab<Real> &L = g.L[p.layer];
    // step size
    {
        const Real mut = L.mua + L.mus;
        if (p.sleft == Real(0)) {
            p.s = -std::log(draw<Real>(rng)) / mut;
        } else {
            p.s = p.sleft / mut;
            p.sleft = Real(0);
        }
    }
    // distance to the boundary along the current direction
    bool hit = false;
    {
        Real db;
        bool moving = true;
        if (p.uz > Real(0)) {
            db = (L.z1 - p.z) / p.uz;
        } else if (p.uz < Real(0)) {
            db = (L.z0 - p.z) / p.uz;
        } else {
            moving = false;
            db = Real(0);
        }
        if (moving && p.s > db) {
            p.sleft = (p.s - db) * (L.mua + L.mus);
            p.s = db;
            hit = true;
        }
    }
    p.x += p.s * p.ux;
    p.y += p.s * p.uy;
    p.z += p.s * p.uz;
    if (hit) {
        ++t.boundary;
        cross(p, g, rng, t);
    } else {
        const Real dwa = p.w * L.mua / (L.mua + L.mus);
        p.w -= dwa;
        t.absorb(p, dwa);
        scatter(p, g.L[p.layer].g, rng);
    }
    if (!p.dead && p.w < K<Real>::wmin) {
        if (p.w == Real(0)) {
            p.dead = true;
        } else if (draw<Real>(rng) < K<Real>::chance) {
            p.w /= K<Real>::chance;
        } else {
            p.dead = true;
        }
    }
}

template <class Real> void one_photon(const Geo<Real> &g, uint64_t seed, uint64_t id, BatchTally<Real> &t) {
    Stream rng(seed, id);
    Packet<Real> p;
    p.x = p.y = p.z = Real(0);
    p.ux = p.uy = Real(0);
    p.uz = Real(1);
    p.w = Real(1) - specular(g);
    p.s = p.sleft = Real(0);
    p.layer = 0;
    p.dead = false;
    while (!p.dead) {
        one_step(p, g, rng, t);
    }
}

// ---------------------------------------------------------------- batches and workers
struct BatchPlan {
    uint64_t base, extra;
    uint64_t count_of(uint64_t b) const { return base + (b < extra ? 1 : 0); }
    uint64_t first_of(uint64_t b) const { return b * base + (b < extra ? b : extra); }
};

struct BatchDone {
    double rd = 0, tt = 0;
    std::vector<double> absorbed, az, rr, arz, rra, tra;
    std::vector<uint64_t> n_arz, n_rra, n_tra;
    uint64_t events = 0, anomalies = 0, boundary = 0;
};

static std::vector<double> values(const std::vector<Neumaier> &v) {
    std::vector<double> o(v.size());
    for (size_t i = 0; i < v.size(); ++i) o[i] = v[i].value();
    return o;
}

template <class Real>
BatchDone run_batch(const Geo<Real> &g, uint64_t seed, uint64_t first, uint64_t count, bool counts) {
    BatchTally<Real> t(g, counts);
    for (uint64_t id = first; id < first + count; ++id) {
        one_photon(g, seed, id, t);
    }
    BatchDone d;
    d.rd = t.rd.value();
    d.tt = t.tt.value();
    d.absorbed = values(t.absorbed);
    d.az = values(t.az);
    d.rr = values(t.rr);
    d.arz = values(t.arz);
    d.rra = values(t.rra);
    d.tra = values(t.tra);
    d.events = t.events;
    d.anomalies = t.anomalies;
    d.boundary = t.boundary;
    d.n_arz = std::move(t.n_arz);
    d.n_rra = std::move(t.n_rra);
    d.n_tra = std::move(t.n_tra);
    return d;
}

}  // namespace oracle

extern "C" {

// Philox4x32-10 of one block (known-answer checks).
void oracle_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    const oracle::Block b = oracle::philox10(oracle::Block{{ctr[0], ctr[1], ctr[2], ctr[3]}}, key[0], key[1]);
    std::memcpy(out, b.v, sizeof b.v);
}

// The first n 32-bit words of photon `id`'s stream under `seed`.
void oracle_stream(uint64_t seed, uint64_t id, uint64_t n, uint32_t *out) {
    oracle::Stream s(seed, id);
    for (uint64_t i = 0; i < n; ++i) out[i] = s.word();
}

// Fresnel reflectance of the walk (precision 32 or 64); returns R and writes cos(transmission).
double oracle_fresnel(int precision, double n1, double n2, double ca1, double *ca2) {
    if (precision == 32) {
        float c2 = 0;
        const float r = oracle::fresnel_r<float>(static_cast<float>(n1), static_cast<float>(n2),
                                                 static_cast<float>(ca1), c2);
        *ca2 = c2;
        return r;
    }
    double c2 = 0;
    const double r = oracle::fresnel_r<double>(n1, n2, ca1, c2);
    *ca2 = c2;
    return r;
}

// Run one .mci run on the CPU. precision: 64 or 32 (transport; tallies are compensated doubles).
// threads: 0 = one per hardware thread, capped at the batch count. Returns 0 on success, 1 on a
// bad argument (message in out->error).
int oracle_run(const oracle_spec *spec, uint64_t photons, int32_t batches, uint64_t seed, int32_t precision,
               int32_t threads, oracle_out *out) {
    using namespace oracle;
    std::memset(out->error, 0, sizeof out->error);
    auto fail = [&](const char *m) {
        std::strncpy(out->error, m, sizeof out->error - 1);
        return 1;
    };
    if (spec->num_layers < 1 || spec->num_layers > kMaxLayers) return fail("num_layers out of range");
    if (batches < 1 || static_cast<uint64_t>(batches) > photons) return fail("bad batch count");
    if (spec->nz < 1 || spec->nr < 1 || spec->na < 1) return fail("bad grid");
    if (precision != 32 && precision != 64) return fail("precision must be 32 or 64");
    const auto t0 = std::chrono::steady_clock::now();
    const bool f32 = precision == 32;
    const Geo<double> g64 = make_geo<double>(*spec);
    const Geo<float> g32 = make_geo<float>(*spec);
    const uint64_t nb = static_cast<uint64_t>(batches);
    const BatchPlan plan{photons / nb, photons % nb};
    int nthreads = threads;
    if (nthreads <= 0) nthreads = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
    if (nthreads > batches) nthreads = batches;
    const bool counts = out->n_a_rz || out->n_rd_ra || out->n_tt_ra;

    std::vector<BatchDone> done(nb);
    std::atomic<uint64_t> next{0};
    std::exception_ptr err;
    std::mutex mu;
    auto worker = [&]() {
        try {
            for (;;) {
                const uint64_t b = next.fetch_add(1, std::memory_order_relaxed);
                if (b >= nb) return;
                done[b] = f32 ? run_batch(g32, seed, plan.first_of(b), plan.count_of(b), counts)
                              : run_batch(g64, seed, plan.first_of(b), plan.count_of(b), counts);
            }
        } catch (...) {
            std::lock_guard<std::mutex> lk(mu);
            if (!err) err = std::current_exception();
            next.store(nb);
        }
    };
    {
        std::vector<std::thread> pool;
        for (int t = 1; t < nthreads; ++t) pool.emplace_back(worker);
        worker();
        for (auto &th : pool) th.join();
    }
    if (err) return fail("worker failed");

    const size_t L = static_cast<size_t>(spec->num_layers);
    const size_t nz = static_cast<size_t>(spec->nz), nr = static_cast<size_t>(spec->nr),
                 na = static_cast<size_t>(spec->na);
    const size_t nrz = nr * nz, nra = nr * na;
    std::fill(out->a_z, out->a_z + nz, 0.0);
    std::fill(out->rd_r, out->rd_r + nr, 0.0);
    std::fill(out->a_rz, out->a_rz + nrz, 0.0);
    std::fill(out->rd_ra, out->rd_ra + nra, 0.0);
    std::fill(out->tt_ra, out->tt_ra + nra, 0.0);
    if (out->n_a_rz) std::fill(out->n_a_rz, out->n_a_rz + nrz, uint64_t(0));
    if (out->n_rd_ra) std::fill(out->n_rd_ra, out->n_rd_ra + nra, uint64_t(0));
    if (out->n_tt_ra) std::fill(out->n_tt_ra, out->n_tt_ra + nra, uint64_t(0));
    // In batch order, as src/cpu/engine.cpp:201-209 merges them.
    for (uint64_t b = 0; b < nb; ++b) {
        const BatchDone &d = done[b];
        out->rd[b] = d.rd;
        out->tt[b] = d.tt;
        for (size_t l = 0; l < L; ++l) out->absorbed[b * L + l] = d.absorbed[l];
        out->events[b] = d.events;
        out->anomalies[b] = d.anomalies;
        if (out->boundary_steps) out->boundary_steps[b] = d.boundary;
        for (size_t i = 0; i < nz; ++i) out->a_z[i] += d.az[i];
        for (size_t i = 0; i < nr; ++i) out->rd_r[i] += d.rr[i];
        for (size_t i = 0; i < nrz; ++i) out->a_rz[i] += d.arz[i];
        for (size_t i = 0; i < nra; ++i) out->rd_ra[i] += d.rra[i];
        for (size_t i = 0; i < nra; ++i) out->tt_ra[i] += d.tra[i];
        if (out->b_a_rz) std::copy(d.arz.begin(), d.arz.end(), out->b_a_rz + b * nrz);
        if (out->b_rd_ra) std::copy(d.rra.begin(), d.rra.end(), out->b_rd_ra + b * nra);
        if (out->b_tt_ra) std::copy(d.tra.begin(), d.tra.end(), out->b_tt_ra + b * nra);
        if (counts) {
            for (size_t i = 0; i < nrz && out->n_a_rz; ++i) out->n_a_rz[i] += d.n_arz[i];
            for (size_t i = 0; i < nra && out->n_rd_ra; ++i) out->n_rd_ra[i] += d.n_rra[i];
            for (size_t i = 0; i < nra && out->n_tt_ra; ++i) out->n_tt_ra[i] += d.n_tra[i];
        }
    }
    out->specular = specular(g64);
    out->threads_used = nthreads;
    out->wall_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return 0;
}
}
