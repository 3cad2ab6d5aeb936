// Formatted text output of the multigrid driver: the residual-history line
// of the .rsd file and the per-cycle screen line of writeResiduals
// (SolverSource/mgnsg3d_mg_par.F90:1449-1516).  The columns and edit
// descriptors are the reference's, so tools that read its .rsd files read
// these:
//   screen (format 501): I7, E14.5, then five times " (" E8.2 ") " E14.5 ...,
//                        then lift and drag as E12.4;
//   .rsd   (format 504): I7, E14.5 x3, then up to 12 x (F13.6, 1X).
// Fortran's Ew.d writes 0.d1..dd E+xx (a leading "0."; a three-digit
// exponent drops the E), Fw.d a fixed field, and a value too wide for its
// field as w asterisks.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>

#include "flite_gpu.h"
#include "flite_prepro.h"

namespace {

// Fortran Ew.d of v, right-justified in w characters
std::string fort_e(double v, int w, int d) {
    std::string body;
    if (!std::isfinite(v)) {
        body = std::isnan(v) ? "NaN" : (v > 0 ? "Infinity" : "-Infinity");
    } else {
        // d significant digits, correctly rounded, as printf writes them
        // (x.yyyyE+zz), then shifted to Fortran's 0.xyyyy form
        char buf[64];
        std::snprintf(buf, sizeof buf, "%.*E", d - 1, std::fabs(v));
        int exp10 = 0;
        std::string digits;
        if (v == 0.0) {
            digits.assign(d, '0');
        } else {
            const char *e = std::strchr(buf, 'E');
            for (const char *q = buf; q < e; ++q)
                if (*q >= '0' && *q <= '9') digits.push_back(*q);
            exp10 = std::atoi(e + 1) + 1;
        }
        char ex[16];
        if (std::abs(exp10) <= 99)
            std::snprintf(ex, sizeof ex, "E%c%02d", exp10 < 0 ? '-' : '+', std::abs(exp10));
        else
            std::snprintf(ex, sizeof ex, "%c%03d", exp10 < 0 ? '-' : '+', std::abs(exp10));
        body = std::string(v < 0 ? "-" : "") + "0." + digits + ex;
    }
    if ((int)body.size() > w) return std::string(w, '*');
    return std::string(w - body.size(), ' ') + body;
}

// Fortran Fw.d of v
std::string fort_f(double v, int w, int d) {
    char buf[512];
    std::snprintf(buf, sizeof buf, "%.*f", d, v);
    std::string body = buf;
    if (!std::isfinite(v)) body = std::isnan(v) ? "NaN" : (v > 0 ? "Infinity" : "-Infinity");
    if ((int)body.size() > w) return std::string(w, '*');
    return std::string(w - body.size(), ' ') + body;
}

std::string fort_i(long v, int w) {
    std::string body = std::to_string(v);
    if ((int)body.size() > w) return std::string(w, '*');
    return std::string(w - body.size(), ' ') + body;
}

int put(char *buf, size_t len, const std::string &s) {
    if (!buf || len < s.size() + 1) return FLITE_EINVAL;
    std::memcpy(buf, s.c_str(), s.size() + 1);
    return FLITE_OK;
}

}  // namespace

extern "C" {

int fp_rsd_line(char *buf, size_t len, int32_t iteration, double res1, double initial_res,
                const double forces[9], const double *res, int32_t nres, int32_t force_calc_type) {
    if (!forces || (nres > 1 && !res) || nres < 1 || nres > 7) return FLITE_EINVAL;
    // currentRes (mg_par:1474-1478): log of the reduction, -100 below 1e-15
    const double cur = (res1 / initial_res > 1.0e-15) ? std::log(res1 / initial_res) : -100.0;
    std::string s = fort_i(iteration, 7) + fort_e(cur / std::log(10.0), 14, 5) + fort_e(forces[0], 14, 5) +
                    fort_e(forces[1], 14, 5);
    // 12(f13.6,1x): latF, frictionDrag, latM, then longM and log10 res(2..nres),
    // or with forceCalcType 3 longMl, longMd, rollM
    double rest[12];
    int n = 0;
    rest[n++] = forces[2];
    rest[n++] = forces[3];
    rest[n++] = forces[4];
    if (force_calc_type == 3) {
        rest[n++] = forces[6];
        rest[n++] = forces[7];
        rest[n++] = forces[8];
    } else {
        rest[n++] = forces[5];
        for (int i = 2; i <= nres; ++i) rest[n++] = std::log(res[i - 1]) / std::log(10.0);
    }
    for (int k = 0; k < n; ++k) s += fort_f(rest[k], 13, 6) + " ";
    return put(buf, len, s);
}

int fp_append_rsd(const char *path, int32_t first, int32_t iteration, double res1, double initial_res,
                  const double forces[9], const double *res, int32_t nres, int32_t force_calc_type) {
    if (!path) return FLITE_EINVAL;
    char line[512];
    int rc = fp_rsd_line(line, sizeof line, iteration, res1, initial_res, forces, res, nres, force_calc_type);
    if (rc != FLITE_OK) return rc;
    // iteration 1 opens the file afresh, later ones append (mg_par:1481-1488)
    std::FILE *f = std::fopen(path, first ? "w" : "a");
    if (!f) return FLITE_EIO;
    const bool ok = std::fprintf(f, "%s\n", line) > 0;
    return (std::fclose(f) == 0 && ok) ? FLITE_OK : FLITE_EIO;
}

int fp_cycle_line(char *buf, size_t len, int32_t iteration, const double res[5], const double maxres[5],
                  double scale, double lift, double drag) {
    if (!res || !maxres) return FLITE_EINVAL;
    std::string s = fort_i(iteration, 7);
    for (int k = 0; k < 5; ++k) s += fort_e(res[k] * scale, 14, 5) + " (" + fort_e(maxres[k], 8, 2) + ") ";
    s += fort_e(lift, 12, 4) + fort_e(drag, 12, 4);
    return put(buf, len, s);
}

}  // extern "C"
