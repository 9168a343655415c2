// The C++ drop-in: tissuemc::cuda_available and tissuemc::run_cuda (TissueMC's
// include/tissuemc/cuda_engine.hpp:9-14) implemented over the C ABI of include/tissuemc_b200.h.
//
// This file only uses the reference's interface names (RunSpec, EngineOptions, RunResult,
// ConfigError), so the same source compiles against TissueMC's own headers in place of
// src/cuda/engine.cu. Error behaviour follows the reference: an invalid run or options throws
// ConfigError, anything else (no device, CUDA failure) std::runtime_error with the message.

#include <cstring>
#include <stdexcept>
#include <vector>

#include "../../../include/tissuemc_b200.h"
#include "b200_options.hpp"
#ifdef TISSUEMC_B200_REFERENCE_HEADERS
// Built inside TissueMC in place of src/cuda/engine.cu: its own headers declare the interface.
#include "tissuemc/config.hpp"
#include "tissuemc/cuda_engine.hpp"
#include "tissuemc/mci.hpp"
#else
#include "tissuemc_api.hpp"
#endif

namespace tissuemc_b200 {

namespace {
uint32_t g_step_cap = 0;
}

void set_step_cap(uint32_t cap) { g_step_cap = cap; }
uint32_t step_cap() { return g_step_cap; }

}  // namespace tissuemc_b200

namespace tissuemc {

namespace {

tmc_run_spec to_c(const RunSpec &run) {
    tmc_run_spec s;
    std::memset(&s, 0, sizeof s);
    s.photons = run.photons;
    s.dz = run.dz;
    s.dr = run.dr;
    s.nz = run.nz;
    s.nr = run.nr;
    s.na = run.na;
    s.n_above = run.n_above;
    s.n_below = run.n_below;
    // more than the maximum is reported by validation; copy what fits
    s.num_layers = static_cast<int32_t>(run.layers.size());
    for (size_t i = 0; i < run.layers.size() && i < TMC_B200_MAX_LAYERS; ++i) {
        const LayerSpec &L = run.layers[i];
        s.layers[i] = tmc_layer{L.n, L.mua, L.mus, L.g, L.d};
    }
    return s;
}

tmc_options to_c(const EngineOptions &o) {
    tmc_options c;
    tmc_b200_default_options(&c);
    c.seed = o.seed;
    c.batches = o.batches;
    c.photons = o.photons;
    c.rung = o.rung;
    c.profiles = o.profiles ? 1 : 0;
    c.step_cap = tissuemc_b200::step_cap();
    return c;
}

[[noreturn]] void raise(const tmc_status &st) {
    if (st.code == TMC_BAD_CONFIG) throw ConfigError(st.message);
    throw std::runtime_error(st.message);
}

}  // namespace

bool cuda_available() { return tmc_b200_available() != 0; }

RunResult run_cuda(const RunSpec &run_in, const EngineOptions &opt) {
    RunSpec run = run_in;
    if (opt.photons != 0) run.photons = opt.photons;
    if (run.layers.size() > static_cast<size_t>(kMaxLayers)) validate(run);  // throws
    const tmc_run_spec spec = to_c(run);
    const tmc_options copt = to_c(opt);
    tmc_status st{};
    tmc_sizes sz{};
    if (tmc_b200_query_sizes(&spec, &copt, &sz, &st) != TMC_OK) raise(st);

    std::vector<uint64_t> first(sz.batches), photons(sz.batches), events(sz.batches), anomalies(sz.batches);
    std::vector<double> rd(sz.batches), tt(sz.batches), absorbed(sz.absorbed);
    RunResult r;
    r.a_z.assign(sz.nz, 0.0);
    r.rd_r.assign(sz.nr, 0.0);
#ifndef TISSUEMC_B200_REFERENCE_HEADERS
    r.tt_r.assign(sz.nr, 0.0);
    r.a_rz.assign(sz.a_rz, 0.0);
    r.rd_ra.assign(sz.ra, 0.0);
    r.tt_ra.assign(sz.ra, 0.0);
#endif
    tmc_result out;
    std::memset(&out, 0, sizeof out);
    out.first_photon = first.data();
    out.photons = photons.data();
    out.rd = rd.data();
    out.tt = tt.data();
    out.absorbed = absorbed.data();
    out.events = events.data();
    out.anomalies = anomalies.data();
    out.a_z = r.a_z.data();
    out.rd_r = r.rd_r.data();
#ifndef TISSUEMC_B200_REFERENCE_HEADERS
    out.tt_r = r.tt_r.data();
    out.a_rz = r.a_rz.data();
    out.rd_ra = r.rd_ra.data();
    out.tt_ra = r.tt_ra.data();
#endif
    if (tmc_b200_run(&spec, &copt, &out, &st) != TMC_OK) raise(st);

    r.spec = run;
    r.engine = "cuda";
    r.precision = "float32";
    r.tally_precision = "fixed64";  // 64-bit fixed-point integer sums
    r.seed = opt.seed;
    r.threads = 1;
    r.rung = opt.rung;
    r.profiles = opt.profiles;
    r.specular = out.specular;
    r.device = out.device;
    r.kernel_seconds = out.kernel_seconds;
    r.wall_seconds = out.wall_seconds;
    const size_t L = sz.layers;
    for (size_t b = 0; b < sz.batches; ++b) {
        BatchResult br;
        br.first_photon = first[b];
        br.photons = photons[b];
        br.rd = rd[b];
        br.tt = tt[b];
        br.absorbed.assign(absorbed.begin() + static_cast<std::ptrdiff_t>(b * L),
                           absorbed.begin() + static_cast<std::ptrdiff_t>((b + 1) * L));
        br.events = events[b];
        br.anomalies = anomalies[b];
        r.batches.push_back(std::move(br));
    }
#ifndef TISSUEMC_B200_REFERENCE_HEADERS
    if (!opt.profiles) {  // the diagnostic reports no profiles at all
        r.tt_r.clear();
        r.a_rz.clear();
        r.rd_ra.clear();
        r.tt_ra.clear();
    }
#endif
    return r;
}

}  // namespace tissuemc
