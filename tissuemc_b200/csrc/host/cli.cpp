// `tissuemc` command line for the B200 engine, with the options, output lines, JSON file and exit
// codes of TissueMC's src/cli/main.cpp:18-204 (exit 1 on anomalies or errors, 2 on usage errors).
//
//   tissuemc --version
//   tissuemc run <input.mci> [--photons N] [--batches B] [--seed S] [--threads T] [--precision P]
//                            [--engine cuda|b200] [--rung N] [--gpu-tally P] [--no-profiles]
//                            [--output FILE] [--mco FILE] [--step-cap N]
//
// --engine defaults to the GPU here: this binary carries the B200 engine only (the reference's CPU
// engine stays the reference's). --threads and --precision are accepted and recorded as the
// reference's GPU engine records them (the transport is float32, one host thread).

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <fstream>
#include <string>

#include "../../../include/tissuemc_b200.h"
#include "b200_options.hpp"
#include "tissuemc_api.hpp"

namespace {

void usage(std::FILE *to) {
    std::fprintf(to,
                 "usage:\n"
                 "  tissuemc --version\n"
                 "  tissuemc run <input.mci> [options]\n"
                 "\n"
                 "options for 'run':\n"
                 "  --photons N    override the photon count in the input file\n"
                 "  --batches B    number of batches for the standard error (default 10)\n"
                 "  --seed S       64-bit random seed (default 1)\n"
                 "  --threads T    accepted for compatibility (the GPU engine uses one host thread)\n"
                 "  --precision P  accepted for compatibility (GPU transport is float32)\n"
                 "  --engine E     cuda or b200 (both: the B200 engine, default)\n"
                 "  --rung N       accepted for compatibility: 0, 1, 3, 5, 6, 7 or 8\n"
                 "  --gpu-tally P  accepted for compatibility (tallies are 64-bit fixed point)\n"
                 "  --no-profiles  diagnostic for rung 6: skip the profile tallies\n"
                 "  --output FILE  write full results as JSON\n"
                 "  --mco FILE     also write each run as an MCML output file (FILE, or FILE's stem\n"
                 "                 with _<run> appended when the input holds several runs)\n"
                 "  --step-cap N   end a packet still alive after N steps and count it as an\n"
                 "                 anomaly (default 2000000000)\n");
}

unsigned long long count_arg(const char *name, const char *text) {
    char *end = nullptr;
    const unsigned long long v = std::strtoull(text, &end, 10);
    if (end == text || *end != '\0' || text[0] == '-') {
        std::fprintf(stderr, "tissuemc: %s expects a non-negative integer, got '%s'\n", name, text);
        std::exit(2);
    }
    return v;
}

// The run as an MCML .mco file through the library's writer (tmc_b200_write_mco).
bool write_mco(const tissuemc::RunSpec &spec, const tissuemc::EngineOptions &opt, const tissuemc::RunResult &res,
               const std::string &path) {
    tmc_run_spec c{};
    c.photons = res.photons();
    c.dz = spec.dz;
    c.dr = spec.dr;
    c.nz = spec.nz;
    c.nr = spec.nr;
    c.na = spec.na;
    c.n_above = spec.n_above;
    c.n_below = spec.n_below;
    c.num_layers = static_cast<int32_t>(spec.layers.size());
    for (size_t l = 0; l < spec.layers.size() && l < TMC_B200_MAX_LAYERS; ++l) {
        const auto &y = spec.layers[l];
        c.layers[l] = tmc_layer{y.n, y.mua, y.mus, y.g, y.d};
    }
    tmc_options o{};
    o.seed = opt.seed;
    o.batches = static_cast<int32_t>(res.batches.size());
    const size_t B = res.batches.size(), L = spec.layers.size();
    std::vector<uint64_t> photons(B);
    std::vector<double> rd(B), tt(B), absorbed(B * L);
    for (size_t b = 0; b < B; ++b) {
        photons[b] = res.batches[b].photons;
        rd[b] = res.batches[b].rd;
        tt[b] = res.batches[b].tt;
        for (size_t l = 0; l < L; ++l) absorbed[b * L + l] = res.batches[b].absorbed[l];
    }
    std::vector<double> a_rz = res.a_rz, rd_ra = res.rd_ra, tt_ra = res.tt_ra;
    tmc_result r{};
    r.photons = photons.data();
    r.rd = rd.data();
    r.tt = tt.data();
    r.absorbed = absorbed.data();
    r.a_rz = a_rz.data();
    r.rd_ra = rd_ra.data();
    r.tt_ra = tt_ra.data();
    r.specular = res.specular;
    r.kernel_seconds = res.kernel_seconds;
    std::snprintf(r.device, sizeof r.device, "%s", res.device.c_str());
    tmc_status st{};
    if (tmc_b200_write_mco(&c, &o, &r, path.c_str(), &st) != TMC_OK) {
        std::fprintf(stderr, "tissuemc: %s\n", st.message);
        return false;
    }
    return true;
}

int run_command(int argc, char **argv) {
    if (argc < 3) {
        usage(stderr);
        return 2;
    }
    const std::string input = argv[2];
    tissuemc::EngineOptions opt;
    std::string output, mco;
    for (int i = 3; i < argc; ++i) {
        const std::string a = argv[i];
        auto value = [&](const char *name) -> const char * {
            if (i + 1 >= argc) {
                std::fprintf(stderr, "tissuemc: %s needs a value\n", name);
                std::exit(2);
            }
            return argv[++i];
        };
        if (a == "--photons") {
            opt.photons = count_arg("--photons", value("--photons"));
        } else if (a == "--batches") {
            opt.batches = static_cast<int>(count_arg("--batches", value("--batches")));
        } else if (a == "--seed") {
            opt.seed = count_arg("--seed", value("--seed"));
        } else if (a == "--threads") {
            opt.threads = static_cast<int>(count_arg("--threads", value("--threads")));
        } else if (a == "--precision") {
            const std::string p = value("--precision");
            if (p != "float64" && p != "float32") {
                std::fprintf(stderr, "tissuemc: --precision must be float64 or float32, got '%s'\n", p.c_str());
                return 2;
            }
            opt.precision = p == "float32" ? tissuemc::Precision::Float32 : tissuemc::Precision::Float64;
        } else if (a == "--engine") {
            const std::string e = value("--engine");
            if (e == "cpu") {
                std::fprintf(stderr, "tissuemc: this binary carries the B200 engine only; the CPU engine "
                                     "is TissueMC's own (use --engine cuda or b200)\n");
                return 2;
            }
            if (e != "cuda" && e != "b200") {
                std::fprintf(stderr, "tissuemc: --engine must be cuda or b200, got '%s'\n", e.c_str());
                return 2;
            }
        } else if (a == "--no-profiles") {
            opt.profiles = false;
        } else if (a == "--rung") {
            opt.rung = static_cast<int>(count_arg("--rung", value("--rung")));
        } else if (a == "--gpu-tally") {
            const std::string p = value("--gpu-tally");
            if (p != "float64" && p != "float32") {
                std::fprintf(stderr, "tissuemc: --gpu-tally must be float64 or float32, got '%s'\n", p.c_str());
                return 2;
            }
        } else if (a == "--output") {
            output = value("--output");
        } else if (a == "--mco") {
            mco = value("--mco");
        } else if (a == "--step-cap") {
            const uint64_t cap = count_arg("--step-cap", value("--step-cap"));
            if (cap == 0 || cap > 0xFFFFFFFFull) {
                std::fprintf(stderr, "tissuemc: --step-cap must be between 1 and 4294967295\n");
                return 2;
            }
            tissuemc_b200::set_step_cap(static_cast<uint32_t>(cap));
        } else {
            std::fprintf(stderr, "tissuemc: unknown option '%s'\n", a.c_str());
            usage(stderr);
            return 2;
        }
    }
    const auto runs = tissuemc::parse_mci_file(input);
    std::ofstream json;
    if (!output.empty()) {
        json.open(output);
        if (!json) {
            std::fprintf(stderr, "tissuemc: cannot write '%s'\n", output.c_str());
            return 1;
        }
        json << "{\"runs\":[";
    }
    int status = 0;
    for (size_t r = 0; r < runs.size(); ++r) {
        const tissuemc::RunResult res = tissuemc::run_cuda(runs[r], opt);
        const auto rd = res.rd(), tt = res.tt(), ab = res.absorbed();
        const auto cons = res.conservation_residual();
        std::printf("run %zu: %llu photons, %zu batches, %.2f s (%s, %s)\n", r + 1,
                    static_cast<unsigned long long>(res.photons()), res.batches.size(), res.wall_seconds,
                    res.engine.c_str(), res.precision.c_str());
        std::printf("  device %s, rung %d, kernel %.3f s, %s totals\n", res.device.c_str(), res.rung,
                    res.kernel_seconds, res.tally_precision.c_str());
        std::printf("  specular R_sp = %.6f\n", res.specular);
        std::printf("  diffuse  R_d  = %.6f +/- %.6f\n", rd.mean, rd.se);
        std::printf("  transmit T_t  = %.6f +/- %.6f\n", tt.mean, tt.se);
        std::printf("  absorbed  A   = %.6f +/- %.6f\n", ab.mean, ab.se);
        std::printf("  conservation residual = %+.2e +/- %.2e\n", cons.mean, cons.se);
        if (res.anomalies() != 0) {
            std::fprintf(stderr,
                         "tissuemc: %llu anomalies (non-finite weight or non-unit direction); results are "
                         "not trustworthy\n",
                         static_cast<unsigned long long>(res.anomalies()));
            status = 1;
        }
        if (json.is_open()) {
            if (r) json << ',';
            tissuemc::write_json(res, json);
        }
        if (!mco.empty()) {
            std::string path = mco;
            if (runs.size() > 1) {
                const size_t dot = mco.rfind('.');
                const size_t slash = mco.rfind('/');
                const bool ext = dot != std::string::npos && (slash == std::string::npos || dot > slash);
                path = (ext ? mco.substr(0, dot) : mco) + "_" + std::to_string(r + 1) + (ext ? mco.substr(dot) : "");
            }
            if (!write_mco(runs[r], opt, res, path)) status = 1;
        }
    }
    if (json.is_open()) {
        json << "]}\n";
        json.flush();
        if (!json) {
            std::fprintf(stderr, "tissuemc: error writing '%s'\n", output.c_str());
            return 1;
        }
    }
    return status;
}

}  // namespace

int main(int argc, char **argv) {
    try {
        if (argc >= 2 && std::strcmp(argv[1], "--version") == 0) {
            std::printf("tissuemc 0.1.0 (B200 engine)\n");
            return 0;
        }
        if (argc >= 2 && std::strcmp(argv[1], "run") == 0) return run_command(argc, argv);
        usage(stderr);
        return 2;
    } catch (const std::exception &e) {
        std::fprintf(stderr, "tissuemc: error: %s\n", e.what());
        return 1;
    }
}
