// Result statistics and JSON output with the layout of TissueMC's src/io/json_out.cpp:9-306.
//
// The estimate of a per-photon mean and its standard error come from the per-batch sums (the
// spread of the per-batch means; NaN with fewer than two batches), as json_out.cpp:37-64 defines
// them. The JSON object keeps every key of the reference, in the reference's order, so existing
// readers (validate.py, cross_engine.py) work unchanged; the 2-D tallies and T_t(r) are appended
// after the reference's last key.

#include <cmath>
#include <cstdio>

#include "tissuemc_api.hpp"

namespace tissuemc {

uint64_t RunResult::photons() const {
    uint64_t n = 0;
    for (const auto &b : batches) n += b.photons;
    return n;
}

uint64_t RunResult::events() const {
    uint64_t n = 0;
    for (const auto &b : batches) n += b.events;
    return n;
}

uint64_t RunResult::anomalies() const {
    uint64_t n = 0;
    for (const auto &b : batches) n += b.anomalies;
    return n;
}

namespace {

template <class F> Estimate per_photon(const std::vector<BatchResult> &bs, F value) {
    double total = 0;
    uint64_t photons = 0;
    for (const auto &b : bs) {
        total += value(b);
        photons += b.photons;
    }
    Estimate e;
    e.mean = total / static_cast<double>(photons);
    const size_t n = bs.size();
    if (n < 2) {
        e.se = std::nan("");
        return e;
    }
    double centre = 0;
    for (const auto &b : bs) centre += value(b) / static_cast<double>(b.photons);
    centre /= static_cast<double>(n);
    double ss = 0;
    for (const auto &b : bs) {
        const double d = value(b) / static_cast<double>(b.photons) - centre;
        ss += d * d;
    }
    e.se = std::sqrt(ss / static_cast<double>(n - 1) / static_cast<double>(n));
    return e;
}

double layers_sum(const BatchResult &b) {
    double s = 0;
    for (double a : b.absorbed) s += a;
    return s;
}

}  // namespace

Estimate RunResult::rd() const { return per_photon(batches, [](const BatchResult &b) { return b.rd; }); }
Estimate RunResult::tt() const { return per_photon(batches, [](const BatchResult &b) { return b.tt; }); }
Estimate RunResult::absorbed() const { return per_photon(batches, layers_sum); }
Estimate RunResult::conservation_residual() const {
    Estimate e = per_photon(batches, [](const BatchResult &b) { return b.rd + b.tt + layers_sum(b); });
    e.mean = e.mean + specular - 1.0;
    return e;
}

namespace {

class Writer {
  public:
    explicit Writer(std::ostream &o) : o_(o) {}
    Writer &raw(const char *s) {
        o_ << s;
        return *this;
    }
    Writer &str(const std::string &s) {
        o_ << '"';
        for (char c : s) {
            if (c == '"' || c == '\\') {
                o_ << '\\' << c;
            } else if (static_cast<unsigned char>(c) < 0x20) {
                char buf[8];
                std::snprintf(buf, sizeof buf, "\\u%04x", static_cast<unsigned>(c));
                o_ << buf;
            } else {
                o_ << c;
            }
        }
        o_ << '"';
        return *this;
    }
    // %.17g round-trips a double; JSON has no NaN or infinity, so those are written as null.
    Writer &num(double v) {
        if (!std::isfinite(v)) {
            o_ << "null";
        } else {
            char buf[40];
            std::snprintf(buf, sizeof buf, "%.17g", v);
            o_ << buf;
        }
        return *this;
    }
    Writer &integer(uint64_t v) {
        o_ << v;
        return *this;
    }
    Writer &key(const char *k) {
        str(k);
        o_ << ':';
        return *this;
    }
    Writer &array(const double *v, size_t n) {
        o_ << '[';
        for (size_t i = 0; i < n; ++i) {
            if (i) o_ << ',';
            num(v[i]);
        }
        o_ << ']';
        return *this;
    }
    Writer &array(const std::vector<double> &v) { return array(v.data(), v.size()); }
    // rows x cols, row-major, as an array of rows
    Writer &matrix(const std::vector<double> &v, size_t rows, size_t cols) {
        o_ << '[';
        for (size_t r = 0; r < rows && r * cols < v.size(); ++r) {
            if (r) o_ << ',';
            array(v.data() + r * cols, cols);
        }
        o_ << ']';
        return *this;
    }
    Writer &estimate(const Estimate &e) {
        o_ << '{';
        key("mean").num(e.mean);
        o_ << ',';
        key("se").num(e.se);
        o_ << '}';
        return *this;
    }

  private:
    std::ostream &o_;
};

}  // namespace

void write_json(const RunResult &run, std::ostream &out) {
    Writer j(out);
    const RunSpec &s = run.spec;
    j.raw("{").key("tissuemc_version").str("0.1.0").raw(",");
    j.key("engine").str(run.engine).raw(",");
    j.key("precision").str(run.precision).raw(",");
    j.key("seed").integer(run.seed).raw(",");
    j.key("threads").integer(static_cast<uint64_t>(run.threads)).raw(",");
    j.key("photons").integer(run.photons()).raw(",");
    j.key("output_name").str(s.output_name).raw(",");
    j.key("n_above").num(s.n_above).raw(",");
    j.key("n_below").num(s.n_below).raw(",");
    j.key("layers").raw("[");
    for (size_t i = 0; i < s.layers.size(); ++i) {
        const LayerSpec &L = s.layers[i];
        j.raw(i ? ",{" : "{");
        j.key("n").num(L.n).raw(",").key("mua").num(L.mua).raw(",").key("mus").num(L.mus).raw(",");
        j.key("g").num(L.g).raw(",").key("d").num(L.d).raw("}");
    }
    j.raw("],");
    j.key("grid").raw("{").key("dz").num(s.dz).raw(",").key("dr").num(s.dr).raw(",");
    j.key("nz").integer(static_cast<uint64_t>(s.nz)).raw(",").key("nr").integer(static_cast<uint64_t>(s.nr));
    j.raw(",").key("na").integer(static_cast<uint64_t>(s.na)).raw("},");
    j.key("specular").num(run.specular).raw(",");
    j.key("wall_seconds").num(run.wall_seconds).raw(",");
    j.key("kernel_seconds").num(run.kernel_seconds).raw(",");
    j.key("device").str(run.device).raw(",");
    j.key("tally_precision").str(run.tally_precision).raw(",");
    j.key("rung").integer(static_cast<uint64_t>(run.rung)).raw(",");
    j.key("profiles").raw(run.profiles ? "true" : "false").raw(",");
    j.key("events").integer(run.events()).raw(",");
    j.key("anomalies").integer(run.anomalies()).raw(",");
    j.key("summary").raw("{");
    j.key("rd").estimate(run.rd()).raw(",");
    j.key("tt").estimate(run.tt()).raw(",");
    j.key("absorbed").estimate(run.absorbed()).raw(",");
    j.key("conservation_residual").estimate(run.conservation_residual()).raw("},");
    j.key("batches").raw("[");
    for (size_t i = 0; i < run.batches.size(); ++i) {
        const BatchResult &b = run.batches[i];
        j.raw(i ? ",{" : "{");
        j.key("first_photon").integer(b.first_photon).raw(",");
        j.key("photons").integer(b.photons).raw(",");
        j.key("rd").num(b.rd).raw(",");
        j.key("tt").num(b.tt).raw(",");
        j.key("absorbed").array(b.absorbed).raw(",");
        j.key("events").integer(b.events).raw(",");
        j.key("anomalies").integer(b.anomalies).raw("}");
    }
    j.raw("],");
    j.key("a_z").array(run.a_z).raw(",");
    j.key("rd_r").array(run.rd_r);
    // additions of this engine
    const size_t nr = static_cast<size_t>(s.nr), nz = static_cast<size_t>(s.nz), na = static_cast<size_t>(s.na);
    if (!run.tt_r.empty()) j.raw(",").key("tt_r").array(run.tt_r);
    if (!run.a_rz.empty()) j.raw(",").key("a_rz").matrix(run.a_rz, nr, nz);
    if (!run.rd_ra.empty()) j.raw(",").key("rd_ra").matrix(run.rd_ra, nr, na);
    if (!run.tt_ra.empty()) j.raw(",").key("tt_ra").matrix(run.tt_ra, nr, na);
    j.raw("}");
}

}  // namespace tissuemc
