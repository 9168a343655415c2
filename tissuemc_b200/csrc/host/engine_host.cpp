// Host side of the C ABI that needs no device: validation, sizes, decoding, defaults.

#include "../engine_host.hpp"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

namespace tmc {

RunShape shape_of(const tmc_run_spec &spec, const tmc_options &opt) {
    RunShape s;
    s.photons = opt.photons != 0 ? opt.photons : spec.photons;
    s.nb = opt.batches;
    s.nl = spec.num_layers;
    s.nz = spec.nz;
    s.nr = spec.nr;
    s.na = spec.na;
    return s;
}

TallyOffsets tally_offsets(const RunShape &sh) {
    TallyOffsets t;
    t.batch = 0;
    t.a_rz = static_cast<size_t>(sh.nb) * static_cast<size_t>(4 + sh.nl);
    t.rd_ra = t.a_rz + static_cast<size_t>(sh.nr) * static_cast<size_t>(sh.nz);
    t.tt_ra = t.rd_ra + static_cast<size_t>(sh.nr) * static_cast<size_t>(sh.na);
    t.total = t.tt_ra + static_cast<size_t>(sh.nr) * static_cast<size_t>(sh.na);
    return t;
}

void validate_run(const tmc_run_spec &spec, const tmc_options &opt) {
    auto fail = [](const std::string &m) { throw ConfigFailure(m); };
    const uint64_t photons = opt.photons != 0 ? opt.photons : spec.photons;
    // include/tissuemc/config.hpp:38-66 (RunSpec validation), in the same order and words
    if (photons == 0) fail("number of photons must be > 0");
    if (!(spec.dz > 0) || !(spec.dr > 0)) fail("dz and dr must be > 0");
    if (spec.nz < 1 || spec.nr < 1 || spec.na < 1) fail("grid bin counts must be >= 1");
    if (!(spec.n_above >= 1.0) || !(spec.n_below >= 1.0)) fail("ambient refractive indices must be >= 1");
    if (spec.num_layers < 1) fail("at least one layer is required");
    if (spec.num_layers > TMC_B200_MAX_LAYERS)
        fail("at most " + std::to_string(TMC_B200_MAX_LAYERS) + " layers are supported");
    for (int i = 0; i < spec.num_layers; ++i) {
        const tmc_layer &L = spec.layers[i];
        const std::string where = "layer " + std::to_string(i + 1) + ": ";
        if (!(L.n >= 1.0)) fail(where + "n must be >= 1");
        if (!(L.mua >= 0) || !(L.mus >= 0)) fail(where + "mua and mus must be >= 0");
        if (!(L.mua + L.mus > 0)) fail(where + "clear layers (mua = mus = 0) are not supported");
        if (!(L.g > -1.0 && L.g < 1.0)) fail(where + "g must be in (-1, 1)");
        if (!(L.d > 0) || !std::isfinite(L.d)) fail(where + "thickness must be finite and > 0");
    }
    // src/cuda/engine.cu:328-350 (options)
    if (opt.batches < 1) fail("batches must be >= 1");
    if (static_cast<uint64_t>(opt.batches) > photons) fail("batches cannot exceed the number of photons");
    const int r = opt.rung;
    if (r != 0 && r != 1 && r != 3 && r != 5 && r != 6 && r != 7 && r != 8)
        fail("rung must be 0, 1, 3, 5, 6, 7 or 8 (rungs 2 and 4 are not built yet)");
    if (!opt.profiles && opt.rung != 6) fail("--no-profiles is a diagnostic for rung 6 only");
    // limits of this engine
    if (photons > TMC_B200_MAX_PHOTONS)
        fail("at most " + std::to_string(TMC_B200_MAX_PHOTONS) +
             " photons per run (64-bit fixed-point tally headroom); split the run");
    const double bins = static_cast<double>(spec.nr) * spec.nz + 2.0 * spec.nr * spec.na +
                        static_cast<double>(opt.batches) * (4 + spec.num_layers);
    if (bins > static_cast<double>(1u << 28)) fail("the tally grid is too large (at most 2^28 tally bins)");
    if (opt.threads_per_block < 0 || opt.threads_per_block > 256 || opt.threads_per_block % 32 != 0)
        fail("threads_per_block must be a multiple of 32 in [32, 256] (0 = planner)");
    if (opt.blocks_per_sm < 0 || opt.blocks_per_sm > 32) fail("blocks_per_sm must be in [0, 32]");
    if (opt.smem_budget < 0) fail("smem_budget must be >= 0");
    if (opt.tile_tz < -1) fail("tile_tz must be >= -1 (0 = planner, -1 = no core tile)");
    if (opt.tile_ra_rows < -1) fail("tile_ra_rows must be >= -1 (0 = planner, -1 = none)");
    if (opt.tile_cross < -1 || opt.tile_cross > 1) fail("tile_cross must be -1, 0 or 1");
}

void decode_tallies(const tmc_run_spec &spec, const tmc_options &opt, const uint64_t *raw,
                    tmc_result &res) {
    const RunShape sh = shape_of(spec, opt);
    const TallyOffsets off = tally_offsets(sh);
    const double k = 1.0 / TMC_B200_FIXED_SCALE;
    const uint64_t nb = static_cast<uint64_t>(sh.nb);
    const uint64_t base = sh.photons / nb, extra = sh.photons % nb;
    const size_t S = static_cast<size_t>(4 + sh.nl);
    for (uint64_t b = 0; b < nb; ++b) {
        res.first_photon[b] = b * base + (b < extra ? b : extra);
        res.photons[b] = base + (b < extra ? 1 : 0);
        const uint64_t *row = raw + off.batch + b * S;
        res.rd[b] = static_cast<double>(row[0]) * k;
        res.tt[b] = static_cast<double>(row[1]) * k;
        res.events[b] = row[2];
        res.anomalies[b] = row[3];
        for (int l = 0; l < sh.nl; ++l) res.absorbed[b * sh.nl + l] = static_cast<double>(row[4 + l]) * k;
    }
    const size_t nz = sh.nz, nr = sh.nr, na = sh.na;
    const uint64_t *arz = raw + off.a_rz, *rdra = raw + off.rd_ra, *ttra = raw + off.tt_ra;
    for (size_t iz = 0; iz < nz; ++iz) {
        uint64_t s = 0;  // exact integer projection
        for (size_t ir = 0; ir < nr; ++ir) s += arz[ir * nz + iz];
        res.a_z[iz] = static_cast<double>(s) * k;
    }
    for (size_t ir = 0; ir < nr; ++ir) {
        uint64_t s = 0, t = 0;
        for (size_t ia = 0; ia < na; ++ia) {
            s += rdra[ir * na + ia];
            t += ttra[ir * na + ia];
        }
        res.rd_r[ir] = static_cast<double>(s) * k;
        if (res.tt_r) res.tt_r[ir] = static_cast<double>(t) * k;
    }
    if (res.a_rz)
        for (size_t i = 0; i < nr * nz; ++i) res.a_rz[i] = static_cast<double>(arz[i]) * k;
    if (res.rd_ra)
        for (size_t i = 0; i < nr * na; ++i) res.rd_ra[i] = static_cast<double>(rdra[i]) * k;
    if (res.tt_ra)
        for (size_t i = 0; i < nr * na; ++i) res.tt_ra[i] = static_cast<double>(ttra[i]) * k;
    if (res.raw) std::memcpy(res.raw, raw, off.total * sizeof(uint64_t));
    // Specular reflectance in double, as the reference reports it (src/cuda/engine.cu:292).
    const double r = (spec.n_above - spec.layers[0].n) / (spec.n_above + spec.layers[0].n);
    res.specular = r * r;
}

}  // namespace tmc

using namespace tmc;

namespace {
void put_status(tmc_status *st, int code, const char *msg) {
    if (!st) return;
    st->code = code;
    std::snprintf(st->message, sizeof st->message, "%s", msg);
}
}  // namespace

extern "C" {

void tmc_b200_default_options(tmc_options *opt) {
    if (!opt) return;
    std::memset(opt, 0, sizeof *opt);
    opt->seed = 1;
    opt->batches = 10;
    opt->photons = 0;
    opt->rung = 0;
    opt->profiles = 1;
    opt->device = 0;
    opt->fast_math = 1;
}

int tmc_b200_query_sizes(const tmc_run_spec *spec, const tmc_options *opt, tmc_sizes *sz,
                         tmc_status *st) {
    put_status(st, TMC_OK, "");
    if (!spec || !opt || !sz) {
        put_status(st, TMC_BAD_ARGUMENT, "NULL argument");
        return TMC_BAD_ARGUMENT;
    }
    try {
        validate_run(*spec, *opt);
    } catch (const ConfigFailure &e) {
        put_status(st, TMC_BAD_CONFIG, e.what());
        return TMC_BAD_CONFIG;
    }
    const RunShape sh = shape_of(*spec, *opt);
    sz->batches = static_cast<uint64_t>(sh.nb);
    sz->layers = static_cast<uint64_t>(sh.nl);
    sz->nz = static_cast<uint64_t>(sh.nz);
    sz->nr = static_cast<uint64_t>(sh.nr);
    sz->na = static_cast<uint64_t>(sh.na);
    sz->absorbed = sz->batches * sz->layers;
    sz->a_rz = sz->nr * sz->nz;
    sz->ra = sz->nr * sz->na;
    sz->tally_words = tally_offsets(sh).total;
    sz->device_words = sz->tally_words + 1;  // + the launch's photon-claim counter
    return TMC_OK;
}

int tmc_b200_decode(const tmc_run_spec *spec, const tmc_options *opt, const uint64_t *raw,
                    tmc_result *res, tmc_status *st) {
    put_status(st, TMC_OK, "");
    if (!spec || !opt || !raw || !res) {
        put_status(st, TMC_BAD_ARGUMENT, "NULL argument");
        return TMC_BAD_ARGUMENT;
    }
    try {
        validate_run(*spec, *opt);
        decode_tallies(*spec, *opt, raw, *res);
    } catch (const ConfigFailure &e) {
        put_status(st, TMC_BAD_CONFIG, e.what());
        return TMC_BAD_CONFIG;
    }
    return TMC_OK;
}

}  // extern "C"
