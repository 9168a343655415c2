// Host-only helpers of the B200 engine: run shape, tally layout, validation and decoding.
// Pure C++ (no CUDA), shared by engine.cu and the host-side C ABI entry points.
#pragma once

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>

#include "../../include/tissuemc_b200.h"

namespace tmc {

// An invalid run or invalid options; carries the text the reference's ConfigError would carry.
class ConfigFailure : public std::runtime_error {
  public:
    using std::runtime_error::runtime_error;
};

struct RunShape {
    uint64_t photons;  // after the options' override
    int nb, nl, nz, nr, na;
};

// Word offsets of the fixed-point tally buffer (one contiguous allocation):
//   batch  [nb * (4 + nl)]  per batch: rd, tt, events, anomalies, absorbed[nl]
//   a_rz   [nr * nz]        A(r,z), r-major
//   rd_ra  [nr * na]        R_d(r,a)
//   tt_ra  [nr * na]        T_t(r,a)
struct TallyOffsets {
    size_t batch, a_rz, rd_ra, tt_ra, total;
};

// Launch and shared-memory plan of one walk (see make_plan in engine.cu).
struct Plan {
    int threads, blocks_per_sm, grid;
    int tr_a, tz_a;     // shared core tile of A(r,z)
    int cross;          // 1: the clamped last row and column of A(r,z) are in shared memory too
    int tr_rd, tr_tt;   // shared rows of R_d(r,a), T_t(r,a)
    int batch_smem;     // per-batch totals in shared memory
};

// What the planner needs to know about the device (cudaDeviceProp fields).
struct DeviceLimits {
    int sms;
    size_t smem_sm, smem_block_optin, reserved;
};

RunShape shape_of(const tmc_run_spec &spec, const tmc_options &opt);
TallyOffsets tally_offsets(const RunShape &sh);

// Throws ConfigFailure with the reference's message for an invalid run or options
// (include/tissuemc/config.hpp:38-66, src/cuda/engine.cu:322-350).
void validate_run(const tmc_run_spec &spec, const tmc_options &opt);

// Decode a raw fixed-point tally buffer into the caller's result arrays.
void decode_tallies(const tmc_run_spec &spec, const tmc_options &opt, const uint64_t *raw,
                    tmc_result &res);

}  // namespace tmc
