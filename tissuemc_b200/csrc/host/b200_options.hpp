// Options of the B200 drop-in that TissueMC's EngineOptions (include/tissuemc/cpu_engine.hpp:18-30)
// has no field for. They are process-wide settings read by run_cuda (run_cuda.cpp) and set by this
// engine's own command line (cli.cpp); a TissueMC build that links run_cuda.cpp never sets them
// and gets the defaults.
#pragma once

#include <cstdint>

namespace tissuemc_b200 {

// Steps after which a packet still alive is ended and counted as an anomaly (0: the engine's
// default, 2e9). A low cap makes the anomaly path fire on purpose (the run then exits 1).
void set_step_cap(uint32_t cap);
uint32_t step_cap();

}  // namespace tissuemc_b200
