// C ABI entry point of the .mci reader (tmc_b200_parse_mci), over tissuemc::parse_mci_file.

#include <cstring>
#include <exception>

#include "../../../include/tissuemc_b200.h"
#include "tissuemc_api.hpp"

extern "C" int tmc_b200_parse_mci(const char *path, tmc_run_spec *runs, int32_t max_runs, int32_t *n_runs,
                                  tmc_status *st) {
    auto status = [&](int code, const char *msg) {
        if (st) {
            st->code = code;
            std::strncpy(st->message, msg, sizeof st->message - 1);
            st->message[sizeof st->message - 1] = '\0';
        }
        return code;
    };
    status(TMC_OK, "");
    if (!path || !n_runs || (max_runs > 0 && !runs)) return status(TMC_BAD_ARGUMENT, "NULL argument");
    try {
        const auto parsed = tissuemc::parse_mci_file(path);
        *n_runs = static_cast<int32_t>(parsed.size());
        for (size_t i = 0; i < parsed.size() && static_cast<int32_t>(i) < max_runs; ++i) {
            const tissuemc::RunSpec &r = parsed[i];
            tmc_run_spec &c = runs[i];
            std::memset(&c, 0, sizeof c);
            c.photons = r.photons;
            c.dz = r.dz;
            c.dr = r.dr;
            c.nz = r.nz;
            c.nr = r.nr;
            c.na = r.na;
            c.n_above = r.n_above;
            c.n_below = r.n_below;
            c.num_layers = static_cast<int32_t>(r.layers.size());
            for (size_t l = 0; l < r.layers.size() && l < TMC_B200_MAX_LAYERS; ++l)
                c.layers[l] = tmc_layer{r.layers[l].n, r.layers[l].mua, r.layers[l].mus, r.layers[l].g, r.layers[l].d};
        }
        return TMC_OK;
    } catch (const std::exception &e) {
        return status(TMC_BAD_CONFIG, e.what());
    }
}
