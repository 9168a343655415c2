// Internal interfaces shared by the CUDA translation units of the engine (not part of the ABI).
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

#include "../../include/tissuemc_b200.h"
#include "walk.cuh"

namespace tmc {

// Layer constants of a validated run in float, in the reference's order of evaluation.
void fill_layers(const tmc_run_spec &spec, LayerC *out);

// Launch weight 1 - R_sp in float (physics.hpp:50-66).
float launch_weight(const tmc_run_spec &spec);

// Run validated single runs back to back on one device and stream, one walk launch each (the
// loop the batched sweep replaces). Returns the device time from the first launch to the end of
// the last. When raw is given, it receives every run's tally buffer concatenated, run c at
// (*offsets)[c] words. Throws std::runtime_error on CUDA failure.
double run_single_loop(const tmc_run_spec *specs, const tmc_options *opts, int n, std::vector<uint64_t> *raw,
                       std::vector<size_t> *offsets);

}  // namespace tmc
