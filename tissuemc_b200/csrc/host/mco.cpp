// MCML-format text output (.mco) of one run: tmc_b200_write_mco.
//
// TissueMC itself writes JSON only (src/io/result.cpp); this writer is an addition for tools that
// read MCML's output format. The file has MCML's sections, keywords and ordering — a version line,
// InParm (photons, grid, layers), RAT (specular, diffuse reflectance, absorbed fraction,
// transmittance), A_l, A_z, Rd_r, Rd_a, Tt_r, Tt_a, A_rz, Rd_ra, Tt_ra — so that a reader keyed on
// those words finds what it expects. Values follow the scaling of the MCML manual (Wang, Jacques
// and Zheng, Comput. Methods Programs Biomed. 47:131-146, 1995):
//
//   radial bin i      annulus area      dA_i = 2 pi (i + 1/2) dr^2          (exactly pi((i+1)^2 - i^2) dr^2)
//   angle bin j       ring solid angle  dO_j = 4 pi sin(a_j) sin(da / 2),   a_j = (j + 1/2) da, da = pi / (2 na)
//   A_l [-]           absorbed weight in layer l / N
//   A_z [1/cm]        sum_r A(r,z) / (N dz)
//   Rd_r, Tt_r [1/cm^2]       sum_a W(r,a) / (N dA_i)
//   Rd_a, Tt_a [1/sr]         sum_r W(r,a) / (N dO_j)
//   A_rz [1/cm^3]             A(r,z) / (N dA_i dz)
//   Rd_ra, Tt_ra [1/(cm^2 sr)]  W(r,a) / (N dA_i dO_j cos a_j)
//
// with N the launched packets and W the weights the engine tallied. Out-of-grid deposits sit in
// the last radial, depth or angle bin, as they do in MCML and in the engine's tallies.

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include "../../../include/tissuemc_b200.h"

namespace {

constexpr double kPi = 3.14159265358979323846;

struct Writer {
    std::FILE *f;
    void line(const char *fmt, ...) __attribute__((format(printf, 2, 3)));
};

void Writer::line(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    std::vfprintf(f, fmt, ap);
    va_end(ap);
    std::fputc('\n', f);
}

// One value per line after a section keyword (1-D arrays).
void column(Writer &w, const char *head, const std::vector<double> &v) {
    w.line("%s", head);
    for (double x : v) w.line("%12.4E", x);
    w.line("%s", "");
}

// A 2-D array, rows r, five values per line, after its comment block and keyword.
void matrix(Writer &w, const char *comment, const char *key, const std::vector<double> &v) {
    w.line("%s", comment);
    w.line("%s", key);
    for (size_t i = 0; i < v.size(); ++i) {
        std::fprintf(w.f, "%12.4E ", v[i]);
        if (i % 5 == 4) std::fputc('\n', w.f);
    }
    if (v.size() % 5) std::fputc('\n', w.f);
    w.line("%s", "");
}

}  // namespace

extern "C" int tmc_b200_write_mco(const tmc_run_spec *spec, const tmc_options *opt, const tmc_result *res,
                                  const char *path, tmc_status *st) {
    auto status = [&](int code, const std::string &msg) {
        if (st) {
            st->code = code;
            std::strncpy(st->message, msg.c_str(), sizeof st->message - 1);
            st->message[sizeof st->message - 1] = '\0';
        }
        return code;
    };
    status(TMC_OK, "");
    if (!spec || !opt || !res || !path) return status(TMC_BAD_ARGUMENT, "NULL argument");
    if (!res->photons || !res->rd || !res->tt || !res->absorbed || !res->a_rz || !res->rd_ra || !res->tt_ra)
        return status(TMC_BAD_ARGUMENT, "the .mco writer needs the batch totals and the 2-D arrays a_rz, rd_ra, tt_ra");
    const int L = spec->num_layers, nz = spec->nz, nr = spec->nr, na = spec->na, B = opt->batches;
    if (L < 1 || L > TMC_B200_MAX_LAYERS || nz < 1 || nr < 1 || na < 1 || B < 1 || !(spec->dz > 0) ||
        !(spec->dr > 0))
        return status(TMC_BAD_CONFIG, "invalid grid, layers or batches");

    double N = 0, rd = 0, tt = 0, absorbed = 0;
    std::vector<double> a_l(L, 0.0);
    for (int b = 0; b < B; ++b) {
        N += static_cast<double>(res->photons[b]);
        rd += res->rd[b];
        tt += res->tt[b];
        for (int l = 0; l < L; ++l) a_l[l] += res->absorbed[static_cast<size_t>(b) * L + l];
    }
    if (!(N > 0)) return status(TMC_BAD_CONFIG, "the result holds no photons");
    for (double &a : a_l) {
        absorbed += a;
        a /= N;
    }

    const double dz = spec->dz, dr = spec->dr, da = kPi / (2.0 * na);
    std::vector<double> area(nr), omega(na), cosa(na);
    for (int i = 0; i < nr; ++i) area[i] = 2.0 * kPi * (i + 0.5) * dr * dr;
    for (int j = 0; j < na; ++j) {
        const double a = (j + 0.5) * da;
        omega[j] = 4.0 * kPi * std::sin(a) * std::sin(0.5 * da);
        cosa[j] = std::cos(a);
    }
    std::vector<double> a_z(nz, 0.0), a_rz(static_cast<size_t>(nr) * nz);
    for (int i = 0; i < nr; ++i)
        for (int k = 0; k < nz; ++k) {
            const double v = res->a_rz[static_cast<size_t>(i) * nz + k];
            a_z[k] += v;
            a_rz[static_cast<size_t>(i) * nz + k] = v / (N * area[i] * dz);
        }
    for (double &v : a_z) v /= N * dz;
    auto angular = [&](const double *W, std::vector<double> &by_r, std::vector<double> &by_a,
                       std::vector<double> &ra) {
        by_r.assign(nr, 0.0);
        by_a.assign(na, 0.0);
        ra.resize(static_cast<size_t>(nr) * na);
        for (int i = 0; i < nr; ++i)
            for (int j = 0; j < na; ++j) {
                const double v = W[static_cast<size_t>(i) * na + j];
                by_r[i] += v;
                by_a[j] += v;
                ra[static_cast<size_t>(i) * na + j] = v / (N * area[i] * omega[j] * cosa[j]);
            }
        for (int i = 0; i < nr; ++i) by_r[i] /= N * area[i];
        for (int j = 0; j < na; ++j) by_a[j] /= N * omega[j];
    };
    std::vector<double> rd_r, rd_a, rd_ra, tt_r, tt_a, tt_ra;
    angular(res->rd_ra, rd_r, rd_a, rd_ra);
    angular(res->tt_ra, tt_r, tt_a, tt_ra);

    std::FILE *f = std::fopen(path, "w");
    if (!f) return status(TMC_BAD_ARGUMENT, std::string("cannot open ") + path + " for writing");
    Writer w{f};
    const char *slash = std::strrchr(path, '/');
    w.line("A1 \t# Version number of the file format.");
    w.line("%s", "");
    w.line("####");
    w.line("# Data categories include: ");
    w.line("# InParm, RAT, ");
    w.line("# A_l, A_z, Rd_r, Rd_a, Tt_r, Tt_a, ");
    w.line("# A_rz, Rd_ra, Tt_ra ");
    w.line("####");
    w.line("%s", "");
    w.line("# Written by the B200 photon-walk engine (%s); kernel time %.6g s, seed %llu.",
           res->device[0] ? res->device : "GPU", res->kernel_seconds, static_cast<unsigned long long>(opt->seed));
    w.line("%s", "");
    w.line("InParm \t\t\t# Input parameters. cm is used.");
    w.line("%s \tA\t\t# output file name, ASCII.", slash ? slash + 1 : path);
    w.line("%.0f \t\t\t# No. of photons", N);
    w.line("%G\t%G\t\t# dz, dr [cm]", dz, dr);
    w.line("%d\t%d\t%d\t# No. of dz, dr, da.", nz, nr, na);
    w.line("%s", "");
    w.line("%d\t\t\t\t\t# Number of layers", L);
    w.line("#n\tmua\tmus\tg\td\t# One line for each layer");
    w.line("%G\t\t\t\t\t# n for medium above", spec->n_above);
    for (int l = 0; l < L; ++l) {
        const tmc_layer &y = spec->layers[l];
        w.line("%G\t%G\t%G\t%G\t%G\t# layer %d", y.n, y.mua, y.mus, y.g, y.d, l + 1);
    }
    w.line("%G\t\t\t\t\t# n for medium below", spec->n_below);
    w.line("%s", "");
    w.line("RAT #Reflectance, absorption, transmission. ");
    w.line("%-14.6G \t#Specular reflectance [-]", res->specular);
    w.line("%-14.6G \t#Diffuse reflectance [-]", rd / N);
    w.line("%-14.6G \t#Absorbed fraction [-]", absorbed / N);
    w.line("%-14.6G \t#Transmittance [-]", tt / N);
    w.line("%s", "");
    column(w, "A_l #Absorption as a function of layer. [-]", a_l);
    column(w, "A_z #A[0], [1],..A[nz-1]. [1/cm]", a_z);
    column(w, "Rd_r #Rd[0], [1],..Rd[nr-1]. [1/cm2]", rd_r);
    column(w, "Rd_a #Rd[0], [1],..Rd[na-1]. [sr-1]", rd_a);
    column(w, "Tt_r #Tt[0], [1],..Tt[nr-1]. [1/cm2]", tt_r);
    column(w, "Tt_a #Tt[0], [1],..Tt[na-1]. [sr-1]", tt_a);
    matrix(w,
           "# A[r][z]. [1/cm3]\n# A[0][0], [0][1],..[0][nz-1]\n# A[1][0], [1][1],..[1][nz-1]\n# ...\n"
           "# A[nr-1][0], [nr-1][1],..[nr-1][nz-1]",
           "A_rz", a_rz);
    matrix(w,
           "# Rd[r][angle]. [1/(cm2sr)].\n# Rd[0][0], [0][1],..[0][na-1]\n# Rd[1][0], [1][1],..[1][na-1]\n"
           "# ...\n# Rd[nr-1][0], [nr-1][1],..[nr-1][na-1]",
           "Rd_ra", rd_ra);
    matrix(w,
           "# Tt[r][angle]. [1/(cm2sr)].\n# Tt[0][0], [0][1],..[0][na-1]\n# Tt[1][0], [1][1],..[1][na-1]\n"
           "# ...\n# Tt[nr-1][0], [nr-1][1],..[nr-1][na-1]",
           "Tt_ra", tt_ra);
    const bool ok = std::ferror(f) == 0;
    if (std::fclose(f) != 0 || !ok) return status(TMC_BAD_ARGUMENT, std::string("error writing ") + path);
    return TMC_OK;
}
