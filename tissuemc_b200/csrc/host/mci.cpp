// MCML .mci reader (format of the MCML manual, chapter 9.1), behaving as TissueMC's
// src/io/mci.cpp:97-183: '#' comments, blank lines skipped, parameters in a fixed order, one
// value count per line, integers where the manual requires them, errors carrying the line number.
// The error texts are part of the interface (tools match on them) and are kept word for word.

#include <cerrno>
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <sstream>

#include "tissuemc_api.hpp"

namespace tissuemc {
namespace {

struct Row {
    int line;
    std::vector<std::string> tok;
};

[[noreturn]] void error_at(int line, const std::string &msg) {
    throw ConfigError("line " + std::to_string(line) + ": " + msg);
}

class Rows {
  public:
    explicit Rows(std::istream &in) {
        std::string text;
        int line = 0;
        while (std::getline(in, text)) {
            ++line;
            const auto hash = text.find('#');
            if (hash != std::string::npos) text.resize(hash);
            std::istringstream ws(text);
            Row r{line, {}};
            for (std::string t; ws >> t;) r.tok.push_back(t);
            if (!r.tok.empty()) rows_.push_back(std::move(r));
        }
    }

    const Row &take(size_t count, const std::string &what) {
        if (at_ >= rows_.size()) {
            error_at(rows_.empty() ? 0 : rows_.back().line, "unexpected end of file, expected " + what);
        }
        const Row &r = rows_[at_++];
        if (r.tok.size() != count) {
            error_at(r.line, what + ": expected " + std::to_string(count) + " value(s), found " +
                                 std::to_string(r.tok.size()));
        }
        return r;
    }

    bool empty() const { return at_ >= rows_.size(); }
    int next_line() const { return rows_[at_].line; }

  private:
    std::vector<Row> rows_;
    size_t at_ = 0;
};

double real_of(const Row &r, size_t i, const std::string &what) {
    const char *s = r.tok[i].c_str();
    char *end = nullptr;
    errno = 0;
    const double v = std::strtod(s, &end);
    if (end == s || *end != '\0' || errno == ERANGE || !std::isfinite(v))
        error_at(r.line, what + ": '" + r.tok[i] + "' is not a finite number");
    return v;
}

long long int_of(const Row &r, size_t i, const std::string &what) {
    const char *s = r.tok[i].c_str();
    char *end = nullptr;
    errno = 0;
    const long long v = std::strtoll(s, &end, 10);
    if (end == s || *end != '\0' || errno == ERANGE) error_at(r.line, what + ": '" + r.tok[i] + "' is not an integer");
    return v;
}

}  // namespace

void validate(const RunSpec &run) {
    auto fail = [](const std::string &m) { throw ConfigError(m); };
    if (run.photons == 0) fail("number of photons must be > 0");
    if (!(run.dz > 0) || !(run.dr > 0)) fail("dz and dr must be > 0");
    if (run.nz < 1 || run.nr < 1 || run.na < 1) fail("grid bin counts must be >= 1");
    if (!(run.n_above >= 1.0) || !(run.n_below >= 1.0)) fail("ambient refractive indices must be >= 1");
    if (run.layers.empty()) fail("at least one layer is required");
    if (run.layers.size() > static_cast<size_t>(kMaxLayers))
        fail("at most " + std::to_string(kMaxLayers) + " layers are supported");
    for (size_t i = 0; i < run.layers.size(); ++i) {
        const LayerSpec &L = run.layers[i];
        const std::string where = "layer " + std::to_string(i + 1) + ": ";
        if (!(L.n >= 1.0)) fail(where + "n must be >= 1");
        if (!(L.mua >= 0) || !(L.mus >= 0)) fail(where + "mua and mus must be >= 0");
        if (!(L.mua + L.mus > 0)) fail(where + "clear layers (mua = mus = 0) are not supported");
        if (!(L.g > -1.0 && L.g < 1.0)) fail(where + "g must be in (-1, 1)");
        if (!(L.d > 0) || !std::isfinite(L.d)) fail(where + "thickness must be finite and > 0");
    }
}

std::vector<RunSpec> parse_mci(std::istream &in) {
    Rows rows(in);
    const Row &ver = rows.take(1, "file version");
    if (real_of(ver, 0, "file version") != 1.0)
        error_at(ver.line, "unsupported file version '" + ver.tok[0] + "' (expected 1.0)");
    const Row &nr_row = rows.take(1, "number of runs");
    const long long nruns = int_of(nr_row, 0, "number of runs");
    if (nruns < 1) error_at(nr_row.line, "number of runs must be >= 1");

    constexpr long long kMaxBins = 1000000;
    std::vector<RunSpec> runs;
    for (long long k = 0; k < nruns; ++k) {
        RunSpec run;
        const Row &out = rows.take(2, "output filename and format");
        run.output_name = out.tok[0];
        if (out.tok[1] != "A") error_at(out.line, "output format must be 'A' (ASCII), found '" + out.tok[1] + "'");
        const Row &np = rows.take(1, "number of photons");
        const long long photons = int_of(np, 0, "number of photons");
        if (photons < 1) error_at(np.line, "number of photons must be >= 1");
        run.photons = static_cast<uint64_t>(photons);
        const Row &step = rows.take(2, "dz and dr");
        run.dz = real_of(step, 0, "dz");
        run.dr = real_of(step, 1, "dr");
        const Row &grid = rows.take(3, "grid counts (nz nr na)");
        const long long nz = int_of(grid, 0, "nz"), nr = int_of(grid, 1, "nr"), na = int_of(grid, 2, "na");
        if (nz < 1 || nr < 1 || na < 1 || nz > kMaxBins || nr > kMaxBins || na > kMaxBins)
            error_at(grid.line, "grid counts must be integers in [1, 1000000]");
        run.nz = static_cast<int>(nz);
        run.nr = static_cast<int>(nr);
        run.na = static_cast<int>(na);
        const Row &nl_row = rows.take(1, "number of layers");
        const long long nl = int_of(nl_row, 0, "number of layers");
        if (nl < 1 || nl > kMaxLayers)
            error_at(nl_row.line, "number of layers must be in [1, " + std::to_string(kMaxLayers) + "]");
        run.n_above = real_of(rows.take(1, "refractive index above"), 0, "n above");
        for (long long i = 0; i < nl; ++i) {
            const Row &lr = rows.take(5, "layer (n mua mus g d)");
            const std::string tag = "layer " + std::to_string(i + 1);
            LayerSpec L;
            L.n = real_of(lr, 0, tag + " n");
            L.mua = real_of(lr, 1, tag + " mua");
            L.mus = real_of(lr, 2, tag + " mus");
            L.g = real_of(lr, 3, tag + " g");
            L.d = real_of(lr, 4, tag + " thickness");
            run.layers.push_back(L);
        }
        const Row &below = rows.take(1, "refractive index below");
        run.n_below = real_of(below, 0, "n below");
        try {
            validate(run);
        } catch (const ConfigError &e) {
            error_at(below.line, std::string("invalid run: ") + e.what());
        }
        runs.push_back(std::move(run));
    }
    if (!rows.empty()) error_at(rows.next_line(), "unexpected extra content after the last run");
    return runs;
}

std::vector<RunSpec> parse_mci_file(const std::string &path) {
    std::ifstream f(path);
    if (!f) throw ConfigError("cannot open '" + path + "'");
    try {
        return parse_mci(f);
    } catch (const ConfigError &e) {
        throw ConfigError(path + ": " + e.what());
    }
}

}  // namespace tissuemc
