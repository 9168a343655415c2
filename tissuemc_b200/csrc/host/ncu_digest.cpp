// ncu_digest: a digest of Nsight Compute counters for the engine's kernels.
//
//   ncu -i capture.ncu-rep --page raw --csv > capture.csv
//   ncu_digest capture.csv [other.csv] [--kernel REGEX]
//
// Reads the raw-page CSV that ncu writes (a header row of metric names, a row of units, one row
// per captured launch), keeps the launches whose kernel name matches --kernel (default: all),
// averages them, and prints markdown tables grouped by what explains a kernel's time: launch
// shape and occupancy, issue efficiency and active lanes per warp, pipe utilisation (FP32 FMA, ALU,
// SFU/XU, tensor), warp stall reasons, shared-memory and atomic traffic, local memory, and the
// L2/DRAM side. With two files the digest is side by side (as TissueMC's
// python/tissuemc_analysis/ncu_profile.py compares two rungs), so a change can be read against
// the capture before it. No reference code: the groups are this engine's own.

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <regex>
#include <sstream>
#include <string>
#include <vector>

namespace {

struct Capture {
    std::string path;
    std::map<std::string, std::string> unit;  // metric -> unit
    std::map<std::string, double> value;      // metric -> mean over the kept launches
    std::vector<std::string> kernels;         // names of the kept launches
};

// One CSV record (RFC 4180 quoting: fields in double quotes, "" for a quote inside).
std::vector<std::string> split_csv(const std::string &line) {
    std::vector<std::string> out;
    std::string cur;
    bool quoted = false;
    for (size_t i = 0; i < line.size(); ++i) {
        const char c = line[i];
        if (quoted) {
            if (c == '"') {
                if (i + 1 < line.size() && line[i + 1] == '"') {
                    cur += '"';
                    ++i;
                } else {
                    quoted = false;
                }
            } else {
                cur += c;
            }
        } else if (c == '"') {
            quoted = true;
        } else if (c == ',') {
            out.push_back(cur);
            cur.clear();
        } else if (c != '\r') {
            cur += c;
        }
    }
    out.push_back(cur);
    return out;
}

bool number(const std::string &text, double &v) {
    std::string t;
    for (char c : text)
        if (c != ',') t += c;
    if (t.empty()) return false;
    char *end = nullptr;
    v = std::strtod(t.c_str(), &end);
    return end && *end == '\0';
}

Capture load(const std::string &path, const std::regex &kernel) {
    std::ifstream in(path);
    if (!in) {
        std::fprintf(stderr, "ncu_digest: cannot read %s\n", path.c_str());
        std::exit(2);
    }
    Capture c;
    c.path = path;
    std::string line;
    std::vector<std::string> header, units;
    // skip ncu's own log lines ("==PROF==" and the like) before the header
    while (std::getline(in, line)) {
        if (!line.empty() && line[0] == '"') {
            header = split_csv(line);
            break;
        }
    }
    if (header.empty()) {
        std::fprintf(stderr, "ncu_digest: %s holds no CSV header\n", path.c_str());
        std::exit(2);
    }
    if (std::getline(in, line)) units = split_csv(line);
    int name_col = -1;
    for (size_t i = 0; i < header.size(); ++i)
        if (header[i] == "Kernel Name") name_col = static_cast<int>(i);
    std::map<std::string, double> sum;
    std::map<std::string, int> count;
    while (std::getline(in, line)) {
        if (line.empty() || line[0] != '"') continue;
        const auto f = split_csv(line);
        if (f.size() != header.size()) continue;
        const std::string name = name_col >= 0 ? f[name_col] : "";
        if (!std::regex_search(name, kernel)) continue;
        c.kernels.push_back(name);
        for (size_t i = 0; i < f.size(); ++i) {
            double v;
            if (number(f[i], v)) {
                sum[header[i]] += v;
                count[header[i]] += 1;
            }
        }
    }
    for (const auto &kv : sum) c.value[kv.first] = kv.second / count[kv.first];
    for (size_t i = 0; i < header.size() && i < units.size(); ++i) c.unit[header[i]] = units[i];
    return c;
}

struct Group {
    const char *title;
    const char *pattern;
    double min_value;  // rows whose values are all below this are dropped (stall reasons)
};

const Group kGroups[] = {
    {"Launch and occupancy",
     "^(gpu__time_duration\\.sum|launch__(grid_size|block_size|registers_per_thread|shared_mem_per_block_dynamic)|"
     "sm__warps_active\\.avg\\.pct_of_peak_sustained_active|sm__cycles_active\\.avg)$",
     -1},
    {"Issue and active lanes",
     "^(smsp__issue_active\\.avg\\.pct_of_peak_sustained_active|smsp__thread_inst_executed_per_inst_executed\\.ratio|"
     "smsp__inst_executed\\.sum|smsp__warps_eligible\\.avg\\.per_cycle_active)$",
     -1},
    {"Pipe utilisation (% of peak while active)",
     "^(sm__pipe_(alu|fma|fmaheavy|fmalite|tensor)_cycles_active\\.avg\\.pct_of_peak_sustained_active|"
     "sm__inst_executed_pipe_(xu|lsu|alu|fma|uniform|cbu|adu)\\.avg\\.pct_of_peak_sustained_active|"
     "sm__pipe_tensor_cycles_active_realtime\\.avg\\.pct_of_peak_sustained_elapsed)$",
     -1},
    {"Warp stalls per issued instruction", "^smsp__average_warps_issue_stalled_.*_per_issue_active\\.ratio$", 0.05},
    {"Shared memory and atomics",
     "^(smsp__inst_executed_op_shared_atom\\.sum|smsp__sass_inst_executed_op_shared_(ld|st)\\.sum|"
     "l1tex__data_pipe_lsu_wavefronts_mem_shared(_op_atom)?\\.sum|l1tex__data_bank_conflicts_pipe_lsu_mem_shared\\.sum|"
     "smsp__inst_executed_op_global_red\\.sum)$",
     -1},
    {"Local memory (register spills)", "^l1tex__t_sectors_pipe_lsu_mem_local_op_(ld|st)\\.sum$", -1},
    {"L2 and DRAM",
     "^(dram__bytes_(read|write)\\.sum|lts__t_sector_hit_rate\\.pct|lts__throughput\\.avg\\.pct_of_peak_sustained_elapsed|"
     "lts__t_sectors_op_(red|atom)\\.sum|dram__throughput\\.avg\\.pct_of_peak_sustained_elapsed)$",
     -1},
};

std::string fmt(double v) {
    char b[64];
    const double a = v < 0 ? -v : v;
    if (a != 0 && (a >= 1e7 || a < 1e-3))
        std::snprintf(b, sizeof b, "%.4g", v);
    else if (a >= 100)
        std::snprintf(b, sizeof b, "%.1f", v);
    else
        std::snprintf(b, sizeof b, "%.3f", v);
    return b;
}

}  // namespace

int main(int argc, char **argv) {
    std::vector<std::string> files;
    std::string kernel = ".*";
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        if (a == "--kernel" && i + 1 < argc) {
            kernel = argv[++i];
        } else if (a == "-h" || a == "--help") {
            std::printf("usage: ncu_digest capture.csv [other.csv] [--kernel REGEX]\n");
            return 0;
        } else {
            files.push_back(a);
        }
    }
    if (files.empty() || files.size() > 2) {
        std::fprintf(stderr, "usage: ncu_digest capture.csv [other.csv] [--kernel REGEX]\n");
        return 2;
    }
    std::regex kre;
    try {
        kre = std::regex(kernel);
    } catch (const std::regex_error &) {
        std::fprintf(stderr, "ncu_digest: bad --kernel expression '%s'\n", kernel.c_str());
        return 2;
    }
    std::vector<Capture> caps;
    for (const auto &f : files) {
        caps.push_back(load(f, kre));
        if (caps.back().kernels.empty()) {
            std::fprintf(stderr, "ncu_digest: no launch in %s matches '%s'\n", f.c_str(), kernel.c_str());
            return 1;
        }
    }
    for (const auto &c : caps)
        std::printf("%s: %zu launch(es) of %s\n", c.path.c_str(), c.kernels.size(), c.kernels.front().c_str());
    std::printf("\n");
    for (const Group &g : kGroups) {
        const std::regex re(g.pattern);
        std::map<std::string, bool> names;
        for (const auto &c : caps)
            for (const auto &kv : c.value)
                if (std::regex_search(kv.first, re)) names[kv.first] = true;
        std::vector<std::string> rows;
        for (const auto &kv : names) {
            bool keep = g.min_value < 0;
            for (const auto &c : caps) {
                const auto it = c.value.find(kv.first);
                if (it != c.value.end() && it->second >= g.min_value) keep = true;
            }
            if (keep) rows.push_back(kv.first);
        }
        if (rows.empty()) continue;
        std::printf("### %s\n\n| metric | unit |", g.title);
        for (size_t i = 0; i < caps.size(); ++i) std::printf(" %s |", i ? "B" : (caps.size() > 1 ? "A" : "value"));
        std::printf("\n|---|---|%s\n", caps.size() > 1 ? "---|---|" : "---|");
        for (const auto &m : rows) {
            std::string unit;
            for (const auto &c : caps) {
                const auto u = c.unit.find(m);
                if (u != c.unit.end() && !u->second.empty()) unit = u->second;
            }
            std::printf("| %s | %s |", m.c_str(), unit.c_str());
            for (const auto &c : caps) {
                const auto it = c.value.find(m);
                std::printf(" %s |", it == c.value.end() ? "-" : fmt(it->second).c_str());
            }
            std::printf("\n");
        }
        std::printf("\n");
    }
    return 0;
}
