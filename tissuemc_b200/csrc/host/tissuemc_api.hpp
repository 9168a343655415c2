// The host-side interface TissueMC's CLI and tools program against, re-declared for this engine.
//
// Names, fields and meanings are those of the reference (paths relative to the TissueMC root):
//   LayerSpec, RunSpec, ConfigError, validate ..... include/tissuemc/config.hpp:14-66
//   Precision, TallyPrecision, EngineOptions ...... include/tissuemc/cpu_engine.hpp:11-30
//   BatchResult, Estimate, RunResult, write_json .. include/tissuemc/result.hpp:15-60
//   parse_mci, parse_mci_file ..................... include/tissuemc/mci.hpp:18-21
//   cuda_available, run_cuda ...................... include/tissuemc/cuda_engine.hpp:9-14
// so that code written against the reference's headers compiles against these unchanged. The
// result gains the 2-D tallies (a_rz, rd_ra, tt_ra) and T_t(r) (tt_r), which the reference lacks;
// its existing fields keep their meaning.
#pragma once

#include <cstdint>
#include <istream>
#include <ostream>
#include <stdexcept>
#include <string>
#include <vector>

namespace tissuemc {

inline constexpr int kMaxLayers = 16;

struct LayerSpec {
    double n;    // refractive index
    double mua;  // absorption coefficient [1/cm]
    double mus;  // scattering coefficient [1/cm]
    double g;    // anisotropy
    double d;    // thickness [cm]
};

struct RunSpec {
    std::string output_name;
    uint64_t photons = 0;
    double dz = 0.01, dr = 0.01;
    int nz = 1, nr = 1, na = 1;  // na: exit-angle bins of R_d(r,a), T_t(r,a)
    double n_above = 1.0, n_below = 1.0;
    std::vector<LayerSpec> layers;
};

class ConfigError : public std::runtime_error {
  public:
    using std::runtime_error::runtime_error;
};

// Throws ConfigError naming the offending field (same checks and words as the reference).
void validate(const RunSpec &run);

enum class Precision { Float64, Float32 };
enum class TallyPrecision { Float64, Float32 };

struct EngineOptions {
    uint64_t seed = 1;
    int batches = 10;
    int threads = 1;
    uint64_t photons = 0;  // if nonzero, overrides the photon count in the run description
    Precision precision = Precision::Float64;            // the GPU transport is float32 regardless
    TallyPrecision gpu_tally = TallyPrecision::Float64;  // B200 tallies are 64-bit fixed point
    int rung = 0;          // accepted for compatibility; every rung runs the B200 kernel
    bool profiles = true;  // false: diagnostic without the profile tallies (rung 6 only)
};

struct BatchResult {
    uint64_t first_photon = 0;
    uint64_t photons = 0;
    double rd = 0;
    double tt = 0;
    std::vector<double> absorbed;
    uint64_t events = 0;
    uint64_t anomalies = 0;
};

struct Estimate {
    double mean = 0;
    double se = 0;  // NaN with fewer than two batches
};

struct RunResult {
    RunSpec spec;
    std::string engine;
    std::string precision;
    uint64_t seed = 0;
    int threads = 1;
    double specular = 0;
    std::vector<BatchResult> batches;
    std::vector<double> a_z;   // absorbed weight per depth bin (all photons)
    std::vector<double> rd_r;  // diffuse reflectance weight per radial bin
    double wall_seconds = 0;
    double kernel_seconds = 0;
    std::string device;
    std::string tally_precision = "float64";
    int rung = 0;
    bool profiles = true;
    // Added by this engine (absent from the reference's result):
    std::vector<double> tt_r;   // [nr]      transmittance weight per radial bin
    std::vector<double> a_rz;   // [nr * nz] absorbed weight per (r, z) bin, r-major
    std::vector<double> rd_ra;  // [nr * na] reflectance weight per (r, exit angle) bin
    std::vector<double> tt_ra;  // [nr * na] transmittance weight per (r, exit angle) bin

    uint64_t photons() const;
    uint64_t events() const;
    uint64_t anomalies() const;
    Estimate rd() const;
    Estimate tt() const;
    Estimate absorbed() const;
    Estimate conservation_residual() const;
};

void write_json(const RunResult &run, std::ostream &out);

std::vector<RunSpec> parse_mci(std::istream &in);
std::vector<RunSpec> parse_mci_file(const std::string &path);

bool cuda_available();
RunResult run_cuda(const RunSpec &run, const EngineOptions &options);

}  // namespace tissuemc
